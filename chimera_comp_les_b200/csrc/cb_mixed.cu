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

namespace {
// Compute_eddy_viscosity_LES (les.c:1523-1567) with constant CS for the mixed
// form, whose SGS terms run in FP32: the same k march as the FP64 kernel
// (EDDY_BX x EDDY_BY columns, three velocity planes in shared memory, the raw
// state of the plane after next copied by cp.async while a plane is
// computed), with u = rhoU / rho, the velocity gradients, |S| and nu_t formed
// in FP32 from the FP32 metric vectors (their w: filter width Delta^2 for csi,
// aj for eta); nu_t is stored in the FP64 plane the stage kernel reads.
// nvert nullptr: no immersed body.
struct Met4 {
  const float4 *m[3];
};
constexpr int EF_BX = 32, EF_BY = 8, EF_PX = EF_BX + 2, EF_PN = EF_PX * (EF_BY + 2);
__global__ void __launch_bounds__(EF_BX *EF_BY)
    eddy_viscosity_mixed_kernel(const DevCfg c, const double *const *qu, const Met4 m4, const double *nvert, double *nut,
                                int kchunk) {
  __shared__ float us[3][3][EF_PN];       // [slot][component][node]
  __shared__ double stq[4][EF_PN];        // raw rho, rhoU, rhoV, rhoW of the plane in flight
  __shared__ unsigned char stv[EF_PN];    // the staged node has a velocity source
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * EF_BX + tx;
  const int i0 = 1 + blockIdx.x * EF_BX, j0 = 1 + blockIdx.y * EF_BY;
  const int kb = 1 + blockIdx.z * kchunk, ke = min(c.mz - 1, kb + kchunk);
  const int i = i0 + tx, j = j0 + ty;
  const bool act = i <= c.mx - 2 && j <= c.my - 2;
  auto issue = [&](int kk) {
    for (int e = tid; e < EF_PN; e += EF_BX * EF_BY) {
      const int ly = e / EF_PX, lx = e - ly * EF_PX;
      const int xi = i0 - 1 + lx, yj = j0 - 1 + ly;
      const bool v = qu != nullptr && xi <= c.mx - 1 && yj <= c.my - 1;
      const long long n = v ? gidx(c, xi, yj, kk) : 0;
      stv[e] = v ? 1 : 0;
#pragma unroll
      for (int f = 0; f < 4; f++) cp_async8(&stq[f][e], v ? qu[f] + n : (const double *)nut, v);
    }
    cp_async_commit();
  };
  auto convert = [&](int s) {
    for (int e = tid; e < EF_PN; e += EF_BX * EF_BY) {
      float u0 = 0.f, u1 = 0.f, u2 = 0.f;
      if (stv[e]) {
        const float ri = 1.f / (float)stq[0][e];
        u0 = c.twod == 1 ? 0.f : (float)stq[1][e] * ri;  // lUcat x = 0 with -twoD 1 (rhs.c:1349)
        u1 = (float)stq[2][e] * ri;
        u2 = (float)stq[3][e] * ri;
      }
      us[s][0][e] = u0;
      us[s][1][e] = u1;
      us[s][2][e] = u2;
    }
  };
  auto stage_sync = [&](int kk) {
    issue(kk);
    cp_async_wait_all();
    __syncthreads();
    convert(kk % 3);
    __syncthreads();
  };
  stage_sync(kb - 1);
  stage_sync(kb);
  issue(kb + 1);
  const int e0 = (ty + 1) * EF_PX + tx + 1;
  const float cs = (float)c.cs_const;
  for (int k = kb; k < ke; k++) {
    // the node's metric vectors of plane k, in flight across the barriers
    const long long n = gidx(c, i, j, k);
    float4 mc = make_float4(0.f, 0.f, 0.f, 0.f), me = mc, mz = mc;
    bool solid = false;
    if (act) {
      mc = __ldg(m4.m[0] + n);
      me = __ldg(m4.m[1] + n);
      mz = __ldg(m4.m[2] + n);
      solid = nvert && __ldg(nvert + n) > 0.1;
    }
    cp_async_wait_all();
    __syncthreads();  // plane k+1 staged; every thread is past plane k-1, whose slot (k+1) % 3 is refilled now
    convert((k + 1) % 3);
    __syncthreads();
    if (k + 1 < ke) issue(k + 2);
    if (!act) continue;
    if (solid) {
      nut[n] = 0.;
      continue;
    }
    const int sm = (k - 1) % 3, s0 = k % 3, sp = (k + 1) % 3;
    float dd[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      dd[a][0] = (us[s0][a][e0 + 1] - us[s0][a][e0 - 1]) * 0.5f;
      dd[a][1] = (us[s0][a][e0 + EF_PX] - us[s0][a][e0 - EF_PX]) * 0.5f;
      dd[a][2] = (us[sp][a][e0] - us[sm][a][e0]) * 0.5f;
    }
    const float m[3][3] = {{mc.x, mc.y, mc.z}, {me.x, me.y, me.z}, {mz.x, mz.y, mz.z}};
    const float ajc = me.w;
    float g[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int x = 0; x < 3; x++) g[a][x] = (dd[a][0] * m[0][x] + dd[a][1] * m[1][x] + dd[a][2] * m[2][x]) * ajc;
    const float Sdd = (2.f / 3.f) * ((g[0][0] + g[1][1]) + g[2][2]);
    const float Sxx = g[0][0] - Sdd, Syy = g[1][1] - Sdd, Szz = g[2][2] - Sdd;
    const float Sxy = 0.5f * (g[0][1] + g[1][0]), Sxz = 0.5f * (g[0][2] + g[2][0]), Syz = 0.5f * (g[1][2] + g[2][1]);
    const float Sabs =
        sqrtf(2.f * (Sxx * Sxx + Syy * Syy + Szz * Szz + 2.f * (Sxy * Sxy + Sxz * Sxz + Syz * Syz)));
    nut[n] = (double)(cs * mc.w * Sabs);  // CS * Delta^2 * |S|
  }
}

int eddy_mixed_kchunk(const DevCfg &c, int sms) {
  static int resident = 0;  // blocks per SM, from the occupancy calculator once per process
  if (resident == 0) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, eddy_viscosity_mixed_kernel, EF_BX * EF_BY, 0) != cudaSuccess ||
        nb < 1)
      nb = 1;
    resident = nb;
  }
  const int nk = c.mz - 2;
  if (nk <= 4) return nk < 1 ? 1 : nk;
  const long long tiles = (long long)((c.mx - 2 + EF_BX - 1) / EF_BX) * ((c.my - 2 + EF_BY - 1) / EF_BY);
  const long long slots = (long long)(sms > 0 ? sms : 1) * resident;
  int best = nk;
  double bc = 1e300;
  for (int kc = 4; kc <= nk; kc++) {  // the fewest whole waves, each chunk paying two extra planes
    const long long blocks = tiles * ((nk + kc - 1) / kc);
    const double cost = (double)((blocks + slots - 1) / slots) * (kc + 2);
    if (cost < bc) { bc = cost; best = kc; }
  }
  return best;
}
}  // namespace

cudaError_t launch_eddy_mixed(const DevCfg &c, const double *const *qu, const float4 *const *met4, const double *nvert,
                              double *nut, int sms, cudaStream_t s) {
  const int kc = eddy_mixed_kchunk(c, sms);
  const Met4 m4{{met4[0], met4[1], met4[2]}};
  const dim3 grid((c.mx - 2 + EF_BX - 1) / EF_BX, (c.my - 2 + EF_BY - 1) / EF_BY, (c.mz - 2 + kc - 1) / kc);
  eddy_viscosity_mixed_kernel<<<grid, dim3(EF_BX, EF_BY), 0, s>>>(c, qu, m4, nvert, nut, kc);
  return cudaGetLastError();
}

cudaError_t launch_mixed_prep(const DevCfg &c, const double *const *met, const double *delta2, const double *aj,
                              float4 *const *met4, double *const *gcl, int grid, cudaStream_t s) {
  mixed_prep_kernel<<<grid, 256, 0, s>>>(c, met, delta2, aj, met4, gcl);
  return cudaGetLastError();
}

}  // namespace cb
