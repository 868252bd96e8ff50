/* A C host replaying the call sequence a reference maintainer adds around
 * RungeKutta (GPU_Setup, GPU_Upload, Flow_Solver_GPU): configure from the
 * reference's options, create a context, FormMetrics on the device from the
 * node coordinates, upload nvert and Q, advance nsteps time steps, read Q
 * and the pressure back.  Only include/chimera_b200.h and the shared
 * library are used.
 *
 *   rk_driver IN OUT les fluxorder s ren ma pr dt nsteps
 *
 * IN: int32 mx, my, mz, then the coordinates (3 doubles per node), nvert
 * (1) and Q (5), AoS natural order.  OUT: Q (5 per node) then P (1 per
 * node).  Exit status: 0, or the failing call's CB_E* code. */
#include <stdio.h>
#include <stdlib.h>

#include "chimera_b200.h"

static int fail(const char *what, int rc, cb_ctx *ctx) {
  fprintf(stderr, "%s failed (%d): %s\n", what, rc, ctx ? cb_last_error(ctx) : "");
  return rc ? rc : 1;
}

int main(int argc, char **argv) {
  if (argc != 11) {
    fprintf(stderr, "usage: %s IN OUT les fluxorder s ren ma pr dt nsteps\n", argv[0]);
    return 1;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) return fail("open input", 1, NULL);
  int m[3];
  if (fread(m, sizeof(int), 3, f) != 3) return fail("read sizes", 1, NULL);
  const size_t n = (size_t)m[0] * m[1] * m[2];
  double *coor = malloc(n * 3 * sizeof(double)), *nv = malloc(n * sizeof(double));
  double *q = malloc(n * 5 * sizeof(double)), *p = malloc(n * sizeof(double));
  if (!coor || !nv || !q || !p) return fail("malloc", 1, NULL);
  if (fread(coor, sizeof(double), n * 3, f) != n * 3 || fread(nv, sizeof(double), n, f) != n ||
      fread(q, sizeof(double), n * 5, f) != n * 5)
    return fail("read arrays", 1, NULL);
  fclose(f);

  cb_config cfg;
  cb_config_default(&cfg, m[0], m[1], m[2]);
  cfg.les = atoi(argv[3]);
  cfg.fluxorder = atoi(argv[4]);
  cfg.s_x = cfg.s_y = cfg.s_z = atof(argv[5]);
  cfg.ren = atof(argv[6]);
  cfg.ma = atof(argv[7]);
  cfg.pr = atof(argv[8]);
  cfg.dt = atof(argv[9]);
  const int nsteps = atoi(argv[10]);

  cb_ctx *ctx = NULL;
  int rc = cb_create(&cfg, &ctx);
  if (rc) return fail("cb_create", rc, ctx);
  if ((rc = cb_set_grid(ctx, coor))) return fail("cb_set_grid", rc, ctx);
  if ((rc = cb_set_nvert(ctx, nv))) return fail("cb_set_nvert", rc, ctx);
  if ((rc = cb_upload_state(ctx, q))) return fail("cb_upload_state", rc, ctx);
  if ((rc = cb_rk_step(ctx, nsteps))) return fail("cb_rk_step", rc, ctx);
  if ((rc = cb_sync(ctx))) return fail("cb_sync", rc, ctx);
  if ((rc = cb_download_state(ctx, q, p))) return fail("cb_download_state", rc, ctx);
  cb_destroy(ctx);

  f = fopen(argv[2], "wb");
  if (!f) return fail("open output", 1, NULL);
  if (fwrite(q, sizeof(double), n * 5, f) != n * 5 || fwrite(p, sizeof(double), n, f) != n)
    return fail("write output", 1, NULL);
  fclose(f);
  free(coor); free(nv); free(q); free(p);
  return 0;
}
