// Definitions of StageLaunch / BatchLaunch (cb_launch.h) for one part of the
// stage-kernel variants, chosen by the compile definitions
//   CB_PART_MIX   0: FP64 parity form (built without FMA contraction, IEEE
//                    division and square root), 1: mixed form (FMA, fast FP32)
//   CB_PART_LES   the LES template value
//   CB_PART_BATCH 0: single-block launches, 1: the batched work queue
// The build compiles this file once per combination, so the template variants
// (flux bits x viscous x no-IBM x RHS mode) compile in parallel.
#include "cb_launch.h"
#include "cb_stage.cuh"

#ifndef CB_PART_MIX
#error "compile with -DCB_PART_MIX=0|1 -DCB_PART_LES=0|1 -DCB_PART_BATCH=0|1"
#endif

namespace cb {

namespace {
#if CB_PART_MIX
using PartR = float;
#else
using PartR = double;
#endif
constexpr bool PART_MIX = CB_PART_MIX != 0, PART_LES = CB_PART_LES != 0;
}  // namespace

#if !CB_PART_BATCH

template <typename R, bool MIX, bool LES>
cudaError_t StageLaunch<R, MIX, LES>::attrs() {
  cudaError_t e = stage_attrs<R, MIX, LES, true, false>();
  if (e == cudaSuccess) e = stage_attrs<R, MIX, LES, false, false>();
  if (e == cudaSuccess) e = stage_attrs<R, MIX, LES, true, true>();
  if (e == cudaSuccess) e = stage_attrs<R, MIX, LES, false, true>();
  return e;
}

namespace {
template <typename R, bool MIX, bool LES, bool VISC, bool RHSM>
void launch_one(const DevCfg &c, const DevFields &F, int istage, double alfa, double beta, double adt, int kchunk,
                int fl, bool nv0, int slots, cudaStream_t s) {
  auto kern = stage_gen_kernel<R, MIX, LES, VISC, RHSM>(fl);
  const bool nv = !RHSM && nv0;
  if constexpr (!RHSM)
    if (nv0) kern = stage_nv0_kernel<R, MIX, LES, VISC>(fl);
  kern<<<stage_grid(c, kchunk, slots, stage_tile_rows(fl)), stage_threads<MIX>(fl), stage_smem_for<R, MIX>(fl, nv), s>>>(
      c, F, istage, alfa, beta, adt, kchunk);
}
}  // namespace

template <typename R, bool MIX, bool LES>
cudaError_t StageLaunch<R, MIX, LES>::launch(const DevCfg &c, const DevFields &F, int istage, double alfa, double beta,
                                             double adt, int kchunk, bool visc, bool rhs_mode, int fl, bool nv0,
                                             int slots, cudaStream_t s) {
  if (rhs_mode) {
    if (visc) launch_one<R, MIX, LES, true, true>(c, F, istage, alfa, beta, adt, kchunk, fl, false, slots, s);
    else launch_one<R, MIX, LES, false, true>(c, F, istage, alfa, beta, adt, kchunk, fl, false, slots, s);
  } else {
    if (visc) launch_one<R, MIX, LES, true, false>(c, F, istage, alfa, beta, adt, kchunk, fl, nv0, slots, s);
    else launch_one<R, MIX, LES, false, false>(c, F, istage, alfa, beta, adt, kchunk, fl, nv0, slots, s);
  }
  return cudaGetLastError();
}

template struct StageLaunch<PartR, PART_MIX, PART_LES>;

#else  // CB_PART_BATCH

namespace {
using BatchKern = void (*)(const BatchBlock *, const int2 *, int, unsigned *, int, double, double, double);

// the persistent kernel for FLUX bits fl: with nv0 the no-IBM variants (Roe,
// WENO5, and with LES the constant-sigma ones), else the general kernel (Roe,
// WENO5)
template <typename R, bool MIX, bool LES, bool VISC, int W>
BatchKern batched_nv0_w(int fl) {
  if constexpr (LES) {
    switch (fl & 7) {
      case 1: return stage_batched_kernel<R, MIX, LES, VISC, true, W | 1>;
      case 2: return stage_batched_kernel<R, MIX, LES, VISC, true, W | 2>;
      case 3: return stage_batched_kernel<R, MIX, LES, VISC, true, W | 3>;
      case 4: return stage_batched_kernel<R, MIX, LES, VISC, true, W | 4>;
      case 5: return stage_batched_kernel<R, MIX, LES, VISC, true, W | 5>;
      default: return stage_batched_kernel<R, MIX, LES, VISC, true, W>;
    }
  } else {
    return (fl & FLUX_ROE) ? stage_batched_kernel<R, MIX, LES, VISC, true, W | 1> : stage_batched_kernel<R, MIX, LES, VISC, true, W>;
  }
}
template <typename R, bool MIX, bool LES, bool VISC>
BatchKern batched_kernel(int fl, bool nv0) {
  if (nv0) {
    switch (fl & (FLUX_W5 | FLUX_PLAIN)) {
      case FLUX_W5: return batched_nv0_w<R, MIX, LES, VISC, FLUX_W5>(fl);
      case FLUX_PLAIN: return batched_nv0_w<R, MIX, LES, VISC, FLUX_PLAIN>(fl);
      case FLUX_W5 | FLUX_PLAIN: return batched_nv0_w<R, MIX, LES, VISC, FLUX_W5 | FLUX_PLAIN>(fl);
      default: return batched_nv0_w<R, MIX, LES, VISC, 0>(fl);
    }
  }
  switch (fl & (FLUX_ROE | FLUX_W5)) {
    case FLUX_ROE: return stage_batched_kernel<R, MIX, LES, VISC, false, FLUX_ROE>;
    case FLUX_W5: return stage_batched_kernel<R, MIX, LES, VISC, false, FLUX_W5>;
    case FLUX_ROE | FLUX_W5: return stage_batched_kernel<R, MIX, LES, VISC, false, FLUX_ROE | FLUX_W5>;
    default: return stage_batched_kernel<R, MIX, LES, VISC, false, 0>;
  }
}
template <typename R, bool MIX, bool LES, bool VISC>
cudaError_t batched_attrs() {
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaSuccess;
  for (int fl : {0, FLUX_ROE, FLUX_W5, FLUX_ROE | FLUX_W5})
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(batched_kernel<R, MIX, LES, VISC>(fl, false), attr, (int)stage_smem_for<R, MIX>(fl, false));
  for (int w : {0, FLUX_W5, FLUX_PLAIN, FLUX_W5 | FLUX_PLAIN})
    for (int fl = 0; fl < (LES ? 6 : 2) && e == cudaSuccess; fl++)
      e = cudaFuncSetAttribute(batched_kernel<R, MIX, LES, VISC>(w | fl, true), attr,
                               (int)stage_smem_for<R, MIX>(w | fl, true));
  return e;
}
}  // namespace

template <typename R, bool MIX, bool LES>
cudaError_t BatchLaunch<R, MIX, LES>::attrs() {
  cudaError_t e = batched_attrs<R, MIX, LES, true>();
  if (e == cudaSuccess) e = batched_attrs<R, MIX, LES, false>();
  return e;
}

template <typename R, bool MIX, bool LES>
cudaError_t BatchLaunch<R, MIX, LES>::launch(const BatchBlock *tab, const int2 *items, int nitems, unsigned *counter,
                                             int istage, double alfa, double beta, double adt, bool visc, int fl,
                                             bool nv0, int ctas, cudaStream_t s) {
  auto kern = visc ? batched_kernel<R, MIX, LES, true>(fl, nv0) : batched_kernel<R, MIX, LES, false>(fl, nv0);
  kern<<<ctas, stage_threads<MIX>(fl), stage_smem_for<R, MIX>(fl, nv0), s>>>(tab, items, nitems, counter, istage, alfa, beta,
                                                                       adt);
  return cudaGetLastError();
}

template struct BatchLaunch<PartR, PART_MIX, PART_LES>;

#endif  // CB_PART_BATCH

}  // namespace cb
