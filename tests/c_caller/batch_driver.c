/* A C host with the reference's multi-block loop (the per-block RungeKutta
 * of solvers.c:246, each block with its own bcs.dat line, init.c:556-559),
 * advanced by the batched context: create it from the reference's options,
 * give every block with a physical face code its codes, FormMetrics on the
 * device from each block's node coordinates, upload each block's Q, wrap the
 * interface blocks onto themselves, advance nsteps time steps, read every
 * block's Q back.  Only include/chimera_b200.h and the shared library are
 * used.
 *
 *   batch_driver IN OUT les fluxorder s ren ma pr dt nsteps
 *
 * IN: int32 nblocks; per block int32 mx, my, mz and 6 face codes; then per
 * block the coordinates (3 doubles per node) and Q (5), AoS natural order.
 * OUT: per block Q (5 per node).  Exit status: 0, or the failing call's
 * CB_E* code. */
#include <stdio.h>
#include <stdlib.h>

#include "chimera_b200.h"

#define MAXB 16

static int fail(const char *what, int rc, cb_batch *b) {
  fprintf(stderr, "%s failed (%d): %s\n", what, rc, b ? cb_batch_last_error(b) : "");
  return rc ? rc : 1;
}

int main(int argc, char **argv) {
  if (argc != 11) {
    fprintf(stderr, "usage: %s IN OUT les fluxorder s ren ma pr dt nsteps\n", argv[0]);
    return 1;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) return fail("open input", 1, NULL);
  int nb = 0;
  if (fread(&nb, sizeof(int), 1, f) != 1 || nb < 1 || nb > MAXB) return fail("read block count", 1, NULL);
  int dims[3 * MAXB], codes[6 * MAXB];
  size_t nn[MAXB];
  for (int k = 0; k < nb; k++) {
    if (fread(dims + 3 * k, sizeof(int), 3, f) != 3 || fread(codes + 6 * k, sizeof(int), 6, f) != 6)
      return fail("read block header", 1, NULL);
    nn[k] = (size_t)dims[3 * k] * dims[3 * k + 1] * dims[3 * k + 2];
  }
  double *coor[MAXB], *q[MAXB];
  for (int k = 0; k < nb; k++) {
    coor[k] = malloc(nn[k] * 3 * sizeof(double));
    q[k] = malloc(nn[k] * 5 * sizeof(double));
    if (!coor[k] || !q[k]) return fail("malloc", 1, NULL);
    if (fread(coor[k], sizeof(double), nn[k] * 3, f) != nn[k] * 3 || fread(q[k], sizeof(double), nn[k] * 5, f) != nn[k] * 5)
      return fail("read arrays", 1, NULL);
  }
  fclose(f);

  cb_config cfg;
  cb_config_default(&cfg, dims[0], dims[1], dims[2]);
  cfg.les = atoi(argv[3]);
  cfg.fluxorder = atoi(argv[4]);
  cfg.s_x = cfg.s_y = cfg.s_z = atof(argv[5]);
  cfg.ren = atof(argv[6]);
  cfg.ma = atof(argv[7]);
  cfg.pr = atof(argv[8]);
  cfg.dt = atof(argv[9]);
  const int nsteps = atoi(argv[10]);

  cb_batch *b = NULL;
  int rc = cb_batch_create(&cfg, nb, dims, &b);
  if (rc) return fail("cb_batch_create", rc, b);
  int interfaces = 0;
  for (int k = 0; k < nb; k++) {
    int coded = 0;
    for (int s = 0; s < 6; s++) coded |= codes[6 * k + s] != 7;
    if (coded) {
      if ((rc = cb_batch_set_bctype(b, k, codes + 6 * k))) return fail("cb_batch_set_bctype", rc, b);
    } else {
      interfaces++;
    }
    if ((rc = cb_batch_set_grid(b, k, coor[k]))) return fail("cb_batch_set_grid", rc, b);
    if ((rc = cb_batch_upload_state(b, k, q[k]))) return fail("cb_batch_upload_state", rc, b);
  }
  if (interfaces && (rc = cb_batch_halo_periodic(b))) return fail("cb_batch_halo_periodic", rc, b);
  if ((rc = cb_batch_rk_step(b, nsteps, 0))) return fail("cb_batch_rk_step", rc, b);
  if ((rc = cb_batch_sync(b))) return fail("cb_batch_sync", rc, b);
  for (int k = 0; k < nb; k++)
    if ((rc = cb_batch_download_state(b, k, q[k]))) return fail("cb_batch_download_state", rc, b);
  cb_batch_destroy(b);

  f = fopen(argv[2], "wb");
  if (!f) return fail("open output", 1, NULL);
  for (int k = 0; k < nb; k++)
    if (fwrite(q[k], sizeof(double), nn[k] * 5, f) != nn[k] * 5) return fail("write output", 1, NULL);
  fclose(f);
  for (int k = 0; k < nb; k++) {
    free(coor[k]);
    free(q[k]);
  }
  return 0;
}
