// Host-side launch interface of the stage kernels (single block and batched)
// and of the mixed form's set-up kernel.
#pragma once
#include <cuda_runtime.h>

#include "cb_common.cuh"
#include "cb_stage.cuh"

namespace cb {

// Grid of a stage-kernel launch: (tile columns in i, in j, k-chunks) for
// kchunk > 0; `slots` CTAs (the resident ones) for the balanced segments of
// kchunk == 0.  by: the tile height of the variant (StageGeo::BY).
inline dim3 stage_grid(const DevCfg &c, int kchunk, int slots, int by = SBY) {
  if (kchunk <= 0) return dim3((unsigned)slots);
  return dim3((c.mx - 2 + SBX - 1) / SBX, (c.my - 2 + by - 1) / by, (c.mz - 2 + kchunk - 1) / kchunk);
}
inline int stage_tile_rows(int fl) { return (fl & FLUX_W5) ? SBY_W5 : SBY; }

// Launchers of the stage kernels, defined in cb_stage_parts.cu.  That file is
// compiled once per (form, LES) pair -- the FP64 parity form without FMA
// contraction, the mixed form with it -- and once more for the batched work
// queue, so the many template variants build in parallel.
//
// fl: FLUX bits (FLUX_ROE, FLUX_W5; the constant-sigma bits apply with nv0
// only); nv0: nvert is zero everywhere, the variant without any nvert test
// (time step only); slots: CTAs of the balanced-segment shape (kchunk 0).
template <typename R, bool MIX, bool LES>
struct StageLaunch {
  static cudaError_t attrs();  // shared-memory opt-in of every variant
  static cudaError_t launch(const DevCfg &c, const DevFields &F, int istage, double alfa, double beta, double adt,
                            int kchunk, bool visc, bool rhs_mode, int fl, bool nv0, int slots, cudaStream_t s);
};
// The persistent multi-block work-queue launch (ctas CTAs).
template <typename R, bool MIX, bool LES>
struct BatchLaunch {
  static cudaError_t attrs();
  static cudaError_t launch(const BatchBlock *tab, const int2 *items, int nitems, unsigned *counter, int istage,
                            double alfa, double beta, double adt, bool visc, int fl, bool nv0, int ctas,
                            cudaStream_t s);
};

// Each (form, LES) instantiation is defined in exactly one object, the part
// built with that form's floating-point flags.  Without these declarations a
// part would also instantiate the other parts' launchers (the inline
// dispatchers below name all of them) and compile their kernels with its own
// flags: an FP64 kernel built with FMA contraction, registered beside the
// right one under the same host symbol.
extern template struct StageLaunch<double, false, false>;
extern template struct StageLaunch<double, false, true>;
extern template struct StageLaunch<float, true, false>;
extern template struct StageLaunch<float, true, true>;
extern template struct BatchLaunch<double, false, false>;
extern template struct BatchLaunch<double, false, true>;
extern template struct BatchLaunch<float, true, false>;
extern template struct BatchLaunch<float, true, true>;

inline cudaError_t stage_attrs_all(bool mix) {
  cudaError_t e = mix ? StageLaunch<float, true, true>::attrs() : StageLaunch<double, false, true>::attrs();
  if (e == cudaSuccess) e = mix ? StageLaunch<float, true, false>::attrs() : StageLaunch<double, false, false>::attrs();
  return e;
}
inline cudaError_t launch_stage_any(bool mix, bool les, const DevCfg &c, const DevFields &F, int istage, double alfa,
                                    double beta, double adt, int kchunk, bool visc, bool rhs_mode, int fl, bool nv0,
                                    int slots, cudaStream_t s) {
  if (mix)
    return les ? StageLaunch<float, true, true>::launch(c, F, istage, alfa, beta, adt, kchunk, visc, rhs_mode, fl, nv0, slots, s)
               : StageLaunch<float, true, false>::launch(c, F, istage, alfa, beta, adt, kchunk, visc, rhs_mode, fl, nv0, slots, s);
  return les ? StageLaunch<double, false, true>::launch(c, F, istage, alfa, beta, adt, kchunk, visc, rhs_mode, fl, nv0, slots, s)
             : StageLaunch<double, false, false>::launch(c, F, istage, alfa, beta, adt, kchunk, visc, rhs_mode, fl, nv0, slots, s);
}
inline cudaError_t batch_attrs_all(bool mix) {
  cudaError_t e = mix ? BatchLaunch<float, true, true>::attrs() : BatchLaunch<double, false, true>::attrs();
  if (e == cudaSuccess) e = mix ? BatchLaunch<float, true, false>::attrs() : BatchLaunch<double, false, false>::attrs();
  return e;
}
inline cudaError_t launch_batched_any(bool mix, bool les, const BatchBlock *tab, const int2 *items, int nitems,
                                      unsigned *counter, int istage, double alfa, double beta, double adt, bool visc,
                                      int fl, bool nv0, int ctas, cudaStream_t s) {
  if (mix)
    return les ? BatchLaunch<float, true, true>::launch(tab, items, nitems, counter, istage, alfa, beta, adt, visc, fl, nv0, ctas, s)
               : BatchLaunch<float, true, false>::launch(tab, items, nitems, counter, istage, alfa, beta, adt, visc, fl, nv0, ctas, s);
  return les ? BatchLaunch<double, false, true>::launch(tab, items, nitems, counter, istage, alfa, beta, adt, visc, fl, nv0, ctas, s)
             : BatchLaunch<double, false, false>::launch(tab, items, nitems, counter, istage, alfa, beta, adt, visc, fl, nv0, ctas, s);
}

// FP32 metric vectors (w: filter width, aj, 0) and the FP64 metric divergence
// (sum over directions of h(+1/2) - h(-1/2)) for the mixed form.
cudaError_t launch_mixed_prep(const DevCfg &c, const double *const *met, const double *delta2, const double *aj,
                              float4 *const *met4, double *const *gcl, int grid, cudaStream_t s);
// Compute_eddy_viscosity_LES with constant CS for the mixed form: FP32
// velocity gradients and |S| from the FP32 metric vectors, nu_t into the FP64
// plane nut (interior nodes); qu: the recorded state (nullptr: zero velocity);
// nvert nullptr: no immersed body.  Defined in cb_mixed.cu.
cudaError_t launch_eddy_mixed(const DevCfg &c, const double *const *qu, const float4 *const *met4, const double *nvert,
                              double *nut, int sms, cudaStream_t s);

}  // namespace cb
