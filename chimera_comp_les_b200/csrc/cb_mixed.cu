// Set-up kernel of the mixed-precision form: the FP32 metric vectors and the
// FP64 metric divergence the stage kernel's FP32 fluxes are restored with
// (see cb_stage.cuh for the shift of the reference state).  The mixed stage
// kernels themselves are built from cb_stage_parts.cu.
#include "cb_launch.h"
#include "cb_stage.cuh"

namespace cb {

namespace {
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

cudaError_t launch_mixed_prep(const DevCfg &c, const double *const *met, const double *delta2, const double *aj,
                              float4 *const *met4, double *const *gcl, int grid, cudaStream_t s) {
  mixed_prep_kernel<<<grid, 256, 0, s>>>(c, met, delta2, aj, met4, gcl);
  return cudaGetLastError();
}

}  // namespace cb
