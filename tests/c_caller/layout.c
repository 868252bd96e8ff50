/* Prints the C layout of the structs include/chimera_b200.h declares, as one
 * JSON object: {"cb_config": {"size": S, "fields": {name: offset, ...}},
 * "cb_ibm_info": {...}}.  Compiled by tests/test_c_caller.py with a plain C99
 * compiler to hold the Python ctypes mirror of those structs to the header. */
#include <stddef.h>
#include <stdio.h>

#include "chimera_b200.h"

#define F(T, m) printf("%s\"%s\": %zu", first ? "" : ", ", #m, offsetof(T, m)), first = 0

int main(void) {
  int first = 1;
  printf("{\"cb_config\": {\"size\": %zu, \"fields\": {", sizeof(cb_config));
  F(cb_config, mx); F(cb_config, my); F(cb_config, mz); F(cb_config, bctype); F(cb_config, les);
  F(cb_config, inviscid); F(cb_config, fluxorder); F(cb_config, eno_order); F(cb_config, central);
  F(cb_config, isothermal); F(cb_config, s_x); F(cb_config, s_y); F(cb_config, s_z); F(cb_config, ren);
  F(cb_config, ma); F(cb_config, pr); F(cb_config, gamma); F(cb_config, dt); F(cb_config, st);
  F(cb_config, cs_const); F(cb_config, ci); F(cb_config, ratio); F(cb_config, precision); F(cb_config, device);
  F(cb_config, calc_sigma); F(cb_config, s_x_min); F(cb_config, s_y_min); F(cb_config, s_z_min);
  F(cb_config, sigma_thrsh); F(cb_config, flux); F(cb_config, max_cs); F(cb_config, twall); F(cb_config, twod);
  F(cb_config, i_homo_filter); F(cb_config, j_homo_filter); F(cb_config, k_homo_filter);
  F(cb_config, testfilter_ik); F(cb_config, visT); F(cb_config, tref); F(cb_config, abc);
  F(cb_config, weno_order);
  first = 1;
  printf("}}, \"cb_ibm_info\": {\"size\": %zu, \"fields\": {", sizeof(cb_ibm_info));
  F(cb_ibm_info, ni); F(cb_ibm_info, nj); F(cb_ibm_info, nk); F(cb_ibm_info, cell);
  F(cb_ibm_info, i1); F(cb_ibm_info, j1); F(cb_ibm_info, k1); F(cb_ibm_info, i2); F(cb_ibm_info, j2);
  F(cb_ibm_info, k2); F(cb_ibm_info, i3); F(cb_ibm_info, j3); F(cb_ibm_info, k3); F(cb_ibm_info, pad);
  F(cb_ibm_info, cr1); F(cb_ibm_info, cr2); F(cb_ibm_info, cr3); F(cb_ibm_info, cs1); F(cb_ibm_info, cs2);
  F(cb_ibm_info, cs3); F(cb_ibm_info, d_s); F(cb_ibm_info, d_i); F(cb_ibm_info, pmin);
  printf("}}}\n");
  return 0;
}
