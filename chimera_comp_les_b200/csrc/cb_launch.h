// Host launchers of the stage kernel, one per translation unit: the FP64
// parity form is compiled without FMA contraction (cb_api.cu), the mixed form
// with it (cb_mixed.cu).
#pragma once
#include <cuda_runtime.h>

#include "cb_common.cuh"
#include "cb_stage.cuh"

namespace cb {

cudaError_t set_stage_attrs_mixed();
// Grid of a stage-kernel launch: (tile columns in i, in j, k-chunks) for
// kchunk > 0; `slots` CTAs (the resident ones) for the balanced segments of
// kchunk == 0.
// by: the tile height of the variant (StageGeo::BY).
inline dim3 stage_grid(const DevCfg &c, int kchunk, int slots, int by = SBY) {
  if (kchunk <= 0) return dim3((unsigned)slots);
  return dim3((c.mx - 2 + SBX - 1) / SBX, (c.my - 2 + by - 1) / by, (c.mz - 2 + kchunk - 1) / kchunk);
}
inline int stage_tile_rows(int fl) { return (fl & FLUX_W5) ? SBY_W5 : SBY; }

// fl: flux bits (FLUX_ROE, FLUX_W5; the constant-sigma bits apply with nv0 only);
// nv0: nvert is zero everywhere, the variant without any nvert test (time step
// only); slots: CTAs of the balanced-segment shape (kchunk 0)
cudaError_t launch_stage_mixed(const DevCfg &c, const DevFields &F, int istage, double alfa, double beta, double adt,
                               int kchunk, bool les, bool visc, bool rhs_mode, int fl, bool nv0, int slots,
                               cudaStream_t s);
// FP32 metric vectors (w: filter width, aj, 0) and the FP64 metric divergence
// (sum over directions of h(+1/2) - h(-1/2)) for the mixed form.
cudaError_t launch_mixed_prep(const DevCfg &c, const double *const *met, const double *delta2, const double *aj,
                              float4 *const *met4, double *const *gcl, int grid, cudaStream_t s);

// Persistent batched stage kernel of the mixed form (multi-block work queue).
struct BatchBlock;
cudaError_t set_batched_attrs_mixed();
cudaError_t launch_batched_mixed(const BatchBlock *tab, const int2 *items, int nitems, unsigned *counter, int istage,
                                 double alfa, double beta, double adt, bool les, bool visc, bool nv0, int ctas,
                                 cudaStream_t s);

}  // namespace cb
