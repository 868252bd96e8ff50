// Mixed-precision form of the stage kernel (FP32 flux arithmetic, FP64 state,
// EOS and RK combination).  Compiled with FMA contraction and fast FP32
// division/sqrt; see cb_stage.cuh for the shift of the reference state.
#include "cb_launch.h"
#include "cb_stage.cuh"

namespace cb {

namespace {
template <bool LES, bool VISC, bool RHSM>
cudaError_t attr1() {
  return stage_attrs<float, true, LES, VISC, RHSM>();
}
template <bool LES, bool VISC, bool RHSM>
void launch1(const DevCfg &c, const DevFields &F, int istage, double alfa, double beta, double adt, int kchunk,
             int fl, bool nv0, int slots, cudaStream_t s) {
  const dim3 grid = stage_grid(c, kchunk, slots, stage_tile_rows(fl));
  auto kern = stage_gen_kernel<float, true, LES, VISC, RHSM>(fl);
  const bool nv = !RHSM && nv0;
  if constexpr (!RHSM)
    if (nv0) kern = stage_nv0_kernel<float, true, LES, VISC>(fl);
  kern<<<grid, stage_threads(fl), stage_smem_for<float, true>(fl, nv), s>>>(c, F, istage, alfa, beta, adt, kchunk);
}

__global__ void mixed_prep_kernel(const DevCfg c, const double *const *met, const double *delta2, const double *aj,
                                  float4 *const *met4, double *const *gcl) {
  const long long total = (long long)c.px * c.py * c.pz;
  const long long nx = c.px, ny = c.py;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const float w[3] = {(float)delta2[t], (float)aj[t], 0.f};
    for (int e = 0; e < 3; e++)
      met4[e][t] = make_float4((float)met[3 * e][t], (float)met[3 * e + 1][t], (float)met[3 * e + 2][t], w[e]);
    const int i = (int)(t % nx) - 2, j = (int)((t / nx) % ny) - 2, k = (int)(t / (nx * ny)) - 2;
    const bool interior = i >= 1 && i <= c.mx - 2 && j >= 1 && j <= c.my - 2 && k >= 1 && k <= c.mz - 2;
    for (int a = 0; a < 3; a++) {
      double s = 0.;
      if (interior) {
        for (int d = c.twod == 1 ? 1 : 0; d < 3; d++) {  // -twoD 1 has no i-faces, so no i share
          const long long sd = gstride(c, d);
          const double *m = met[3 * d + a];
          const double hp = 0.5 * (m[t] + m[t + sd]), hm = 0.5 * (m[t - sd] + m[t]);
          s += hp - hm;
        }
      }
      gcl[a][t] = s;
    }
  }
}
}  // namespace

cudaError_t set_stage_attrs_mixed() {
  cudaError_t e;
  if ((e = attr1<true, true, false>()) != cudaSuccess) return e;
  if ((e = attr1<true, false, false>()) != cudaSuccess) return e;
  if ((e = attr1<false, true, false>()) != cudaSuccess) return e;
  if ((e = attr1<false, false, false>()) != cudaSuccess) return e;
  if ((e = attr1<true, true, true>()) != cudaSuccess) return e;
  if ((e = attr1<true, false, true>()) != cudaSuccess) return e;
  if ((e = attr1<false, true, true>()) != cudaSuccess) return e;
  return attr1<false, false, true>();
}

cudaError_t launch_stage_mixed(const DevCfg &c, const DevFields &F, int istage, double alfa, double beta, double adt,
                               int kchunk, bool les, bool visc, bool rhs_mode, int fl, bool nv0, int slots,
                               cudaStream_t s) {
  if (rhs_mode) {
    if (les && visc) launch1<true, true, true>(c, F, istage, alfa, beta, adt, kchunk, fl, false, slots, s);
    else if (les) launch1<true, false, true>(c, F, istage, alfa, beta, adt, kchunk, fl, false, slots, s);
    else if (visc) launch1<false, true, true>(c, F, istage, alfa, beta, adt, kchunk, fl, false, slots, s);
    else launch1<false, false, true>(c, F, istage, alfa, beta, adt, kchunk, fl, false, slots, s);
  } else {
    if (les && visc) launch1<true, true, false>(c, F, istage, alfa, beta, adt, kchunk, fl, nv0, slots, s);
    else if (les) launch1<true, false, false>(c, F, istage, alfa, beta, adt, kchunk, fl, nv0, slots, s);
    else if (visc) launch1<false, true, false>(c, F, istage, alfa, beta, adt, kchunk, fl, nv0, slots, s);
    else launch1<false, false, false>(c, F, istage, alfa, beta, adt, kchunk, fl, nv0, slots, s);
  }
  return cudaGetLastError();
}

namespace {
template <bool LES, bool VISC>
cudaError_t battr1() {
  const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(stage_batched_kernel<float, true, LES, VISC>, a, (int)STAGE_SMEM_BYTES_MIXED);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(stage_batched_kernel<float, true, LES, VISC, true>, a,
                              (int)stage_smem<float, true, true>());
}
template <bool LES, bool VISC>
void blaunch1(const BatchBlock *tab, const int2 *items, int nitems, unsigned *counter, int istage, double alfa,
              double beta, double adt, bool nv0, int ctas, cudaStream_t s) {
  auto kern = nv0 ? stage_batched_kernel<float, true, LES, VISC, true> : stage_batched_kernel<float, true, LES, VISC, false>;
  const size_t smem = nv0 ? stage_smem<float, true, true>() : STAGE_SMEM_BYTES_MIXED;
  kern<<<ctas, SNT, smem, s>>>(tab, items, nitems, counter, istage, alfa, beta, adt);
}
}  // namespace

cudaError_t set_batched_attrs_mixed() {
  cudaError_t e;
  if ((e = battr1<true, true>()) != cudaSuccess) return e;
  if ((e = battr1<true, false>()) != cudaSuccess) return e;
  if ((e = battr1<false, true>()) != cudaSuccess) return e;
  return battr1<false, false>();
}

cudaError_t launch_batched_mixed(const BatchBlock *tab, const int2 *items, int nitems, unsigned *counter, int istage,
                                 double alfa, double beta, double adt, bool les, bool visc, bool nv0, int ctas,
                                 cudaStream_t s) {
  if (les && visc) blaunch1<true, true>(tab, items, nitems, counter, istage, alfa, beta, adt, nv0, ctas, s);
  else if (les) blaunch1<true, false>(tab, items, nitems, counter, istage, alfa, beta, adt, nv0, ctas, s);
  else if (visc) blaunch1<false, true>(tab, items, nitems, counter, istage, alfa, beta, adt, nv0, ctas, s);
  else blaunch1<false, false>(tab, items, nitems, counter, istage, alfa, beta, adt, nv0, ctas, s);
  return cudaGetLastError();
}

cudaError_t launch_mixed_prep(const DevCfg &c, const double *const *met, const double *delta2, const double *aj,
                              float4 *const *met4, double *const *gcl, int grid, cudaStream_t s) {
  mixed_prep_kernel<<<grid, 256, 0, s>>>(c, met, delta2, aj, met4, gcl);
  return cudaGetLastError();
}

}  // namespace cb
