// Device-side definitions shared by the kernels of libchimera_b200.so.
//
// HBM layout (one block of the reference's DMDA):
//   every field is its own plane (SoA) over the padded node box
//   px x (my+4) x (mz+4), node (i,j,k) at ((k+2)*(my+4) + (j+2))*px + (i+2),
//   i in [-2, mx+1].  px = mx+4 rounded up to a multiple of 16 doubles so each
//   row starts on a 128-byte boundary.  The two ghost layers of a periodic
//   direction hold the DMDA wrap-around images (local index -1 -> m-1,
//   -2 -> m-2, m -> 0, m+1 -> 1), exactly what DMGlobalToLocal gives the
//   reference (init.c:156 stencil width 2).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cb {

// Status bits of the sticky device status word.
enum : unsigned { ST_NONFINITE = 1u, ST_NEG_RHO = 2u, ST_NEG_P = 4u };

struct DevCfg {
  int mx, my, mz;
  int px, py, pz;          // padded extents (px = row pitch in doubles)
  long long plane;         // px*py*pz doubles per field
  int bctype[6];
  int les, inviscid, fluxorder, eno_order, central, isothermal;
  double s_x, s_y, s_z;
  double ren, ma, pr, gamma, dt, st, cs_const, ci, ratio;
  double inv_ren;       // 1./ren
  double inv_ren_half;  // 1./ren*0.5
  double gm1;           // gamma-1.0
  double kheat;         // gamma / Pr / (gamma - 1): the mixed form's heat-flux factor
  // mixed form: reference state subtracted before FP32 rounding
  double p_ref, e_ref, t_ref, h_ref;  // h_ref = e_ref + p_ref
  // 1: every nvert value is k/4 with 0 <= k <= 255, so the stage kernel keeps
  // nvert as one exact byte per node in shared memory; 0: read from global
  int nvq;
  // LES shock sensor (rhs.c:3333-3433): hybrid weights from per-node planes
  int calc_sigma;
  double s_x_min, s_y_min, s_z_min, ks;
  int abc;  // -ABC: raw sensor weights 0 above plane k = abc (0: off)
  int flux;  // 0 Rusanov (the reference's), 1 Roe with Harten's entropy fix
  double twall;  // -Twall of the characteristic isothermal wall
  int twod;      // -twoD (1 drops that wall's x velocity term)
  // -visT: Sutherland's law nu = sut_k1 / (Tr + sut_k2) * Tr^1.5 on the face
  // temperature Tr = gm2 * (p0 + p1) / (rho0 + rho1) (rhs.c:1627-1637)
  int sutherland;
  double sut_k1;  // 1./ren*(1+C/Tref), C = 110.4 (rhs.c:1410)
  double sut_k2;  // C/Tref
  double gm2;     // gamma*Ma*Ma
};

// The Sutherland constants of DevCfg from the options, in the reference's
// evaluation order.
inline void set_sutherland(DevCfg &d, int visT, double tref, double ren, double gamma, double ma) {
  const double C_sutherland = 110.4;
  d.sutherland = visT != 0;
  d.sut_k1 = 1. / ren * (1 + C_sutherland / tref);
  d.sut_k2 = C_sutherland / tref;
  d.gm2 = gamma * ma * ma;
}

// Host check of an nvert array for the byte code of DevCfg::nvq.
inline int nvert_codes_exact(const double *nv, size_t n) {
  for (size_t t = 0; t < n; t++) {
    const double c = nv[t] * 4.0;
    if (!(c >= 0.0 && c <= 255.0) || c != (double)(long long)c) return 0;
  }
  return 1;
}

struct DevFields {
  const double *q[5];      // stage input (ghosted)
  const double *qold[5];   // Qold
  double *qout[5];         // stage output
  const double *met[3][3]; // met[0]=csi, met[1]=eta, met[2]=zet; [component]
  const double *aj;
  const double *nvert;
  const double *nut;
  const double *delta2;    // LES filter width squared, pow(pow(1/aj,1/3),2), per node
  // mixed form: FP32 metric vectors, one 16-byte load per node and direction;
  // w carries the FP32 filter width (csi), aj (eta), 0 (zet)
  const float4 *met4[3];
  const double *gcl[3];      // mixed form: per-node metric divergence sum_d dh_d (FP64)
  const double *sig[3];    // hybrid weights per node (only with the shock sensor)
  double *rhs[5];          // formRHS output (rhs mode only)
  unsigned *status;        // sticky status word
  // the pressure lP to read instead of the EqOfState of q (the first stage
  // after an immersed step, whose FormBCS(user, 0) is followed by no
  // EqOfState; the FP64 stage kernel and FormBCS read it); nullptr: EqOfState of q
  const double *pin;
  // node coordinates x, y (the k-lo inflow codes 52 and 47 read them) and the
  // step index user->ti of the running step (code 47), or nullptr
  const double *cx, *cy;
  const int *ti;
};

// 8-byte asynchronous global -> shared copy (valid false: zero-fill, nothing read)
__device__ __forceinline__ void cp_async8(void *sdst, const void *gsrc, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  const int sz = valid ? 8 : 0;  // src-size 0 zero-fills the destination
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(sz) : "memory");
}
// 16-byte asynchronous global -> shared copy through L2 only (both addresses
// 16-byte aligned; valid false: zero-fill, nothing read)
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// brings the line holding p toward this SM's L1 (a hint: nothing is returned)
__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];\n" ::"l"(p)); }
// brings the line holding p into L2 (a hint: nothing is returned)
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__host__ __device__ __forceinline__ long long gidx(const DevCfg &c, int i, int j, int k) {
  return ((long long)(k + 2) * c.py + (j + 2)) * (long long)c.px + (i + 2);
}

__host__ __device__ __forceinline__ long long gstride(const DevCfg &c, int d) {
  return d == 0 ? 1LL : (d == 1 ? (long long)c.px : (long long)c.px * c.py);
}

__device__ __forceinline__ double ldg(const double *p) { return __ldg(p); }

// Hybrid weight sigma of direction d at node (i,j,k): from the sensor's
// planes when it is on; otherwise (rhs.c:3322-3441) every node starts at
// (s_x, s_y, s_z) and interior nodes then take y = z = min(z, y).  Ghost
// nodes carry the wrap-around image.
__device__ __forceinline__ double sigma_at(const DevCfg &c, const DevFields &F, int d, int i, int j, int k) {
  if (c.calc_sigma) return ldg((d == 0 ? F.sig[0] : (d == 1 ? F.sig[1] : F.sig[2])) + gidx(c, i, j, k));
  if (d == 0) return c.s_x;
  if (c.s_y == c.s_z) return c.s_y;  // min(s_z, s_y) = s_y = s_z: the node's position does not matter
  // wrap ghost indices to their owned image (periodic directions only reach ghosts)
  int ii = i < 0 ? i + c.mx : (i >= c.mx ? i - c.mx : i);
  int jj = j < 0 ? j + c.my : (j >= c.my ? j - c.my : j);
  int kk = k < 0 ? k + c.mz : (k >= c.mz ? k - c.mz : k);
  bool interior = ii > 0 && ii < c.mx - 1 && jj > 0 && jj < c.my - 1 && kk > 0 && kk < c.mz - 1;
  if (interior) return c.s_z < c.s_y ? c.s_z : c.s_y;
  return d == 1 ? c.s_y : c.s_z;
}

}  // namespace cb
