// cb_rhs_noalloc: formRHS for callers that cannot allocate device memory.
//
// Some host codes run where they may not call cudaMalloc: a solver inside a
// memory pool owned by another framework, a plugin whose host forbids device
// allocation after start-up, or a rank that must keep its footprint fixed.
// They hand in device arrays they already own and get the RHS back in device
// memory they own.  Everything this computation needs beyond those inputs
// and that output -- the padded SoA planes of the state, metrics, mask, eddy
// viscosity, filter width and RHS, plus a pointer table -- lives in the
// file-scope __device__ arrays below (in an anonymous namespace: internal to
// this translation unit).  They are part of this file's device module: once
// the module is loaded on a GPU (on first use of a kernel of the library under
// CUDA's default lazy loading, at start-up with CUDA_MODULE_LOADING=EAGER) that
// GPU holds them (about 20 MB) until the process exits.
//
// Sharing: every call uses the same arrays and they keep the last call's
// contents.  Calls that overlap on the GPU (different streams or threads)
// race on them; serialise calls, e.g. one stream.
//
// Set-up: every call, with the caller's device current, looks up the arrays'
// device addresses with cudaGetSymbolAddress (no allocation).  The first call
// on a device, and the first after a device reset moved the arrays, also opts
// the RHS kernels into their shared memory; make that first call before any
// stream capture.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/chimera_b200.h"
#include "cb_aux.cuh"
#include "cb_common.cuh"
#include "cb_stage.cuh"

using namespace cb;

namespace {

constexpr int NA_NPLANES = 26;  // Q 5, metrics 9, aj, nvert, nu_t, filter width, RHS 5, coordinates 3
enum { NA_Q = 0, NA_MET = 5, NA_AJ = 14, NA_NVERT = 15, NA_NUT = 16, NA_DELTA2 = 17, NA_RHS = 18, NA_COOR = 23 };

__device__ __align__(256) double na_scratch[(size_t)NA_NPLANES * CB_NOALLOC_MAX_PLANE];
__device__ __align__(256) double *na_ptab[32];

struct NaPtrs {
  double *p[32];
};

__global__ void na_set_ptab(NaPtrs v) {
  if (threadIdx.x < 32) na_ptab[threadIdx.x] = v.p[threadIdx.x];
}

struct NaDevice {
  bool ready = false;
  double *scratch = nullptr;
  double **ptab = nullptr;
};
NaDevice g_dev[64];

template <bool LES, bool VISC>
cudaError_t na_attr() {
  return cudaFuncSetAttribute(stage_kernel<double, false, LES, VISC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)STAGE_SMEM_BYTES);
}

template <bool LES, bool VISC>
void na_launch_rhs(const DevCfg &dc, const DevFields &F, int kchunk, cudaStream_t s) {
  const int nkin = dc.mz - 2;
  dim3 grid((dc.mx - 2 + SBX - 1) / SBX, (dc.my - 2 + SBY - 1) / SBY, (nkin + kchunk - 1) / kchunk);
  stage_kernel<double, false, LES, VISC, true><<<grid, StageThreads<0, false>::N, STAGE_SMEM_BYTES, s>>>(dc, F, 0, 0., 0., 0., kchunk);
}

int na_fail(int code, const char *msg) {
  fprintf(stderr, "chimera_b200: cb_rhs_noalloc: %s\n", msg);
  return code;
}

}  // namespace

extern "C" int cb_rhs_noalloc(const cb_config *cfg, const double *d_coor, const double *d_q, const double *d_nvert,
                              const double *d_nut, double *d_rhs, void *stream) {
  if (!cfg || !d_coor || !d_q || !d_nvert || !d_rhs) return na_fail(CB_E_ARG, "null argument");
  if (cfg->mx < 5 || cfg->my < 5 || cfg->mz < 5) return na_fail(CB_E_ARG, "grid must have at least 5 nodes per direction");
  for (int b = 0; b < 6; b++)
    if (cfg->bctype[b] != 7) return na_fail(CB_E_UNSUPPORTED, "only fully periodic blocks (bctype 7) are built");
  if (cfg->fluxorder < 1 || cfg->fluxorder > 3 || (cfg->eno_order != 2 && cfg->eno_order != 3) ||
      (cfg->les != 0 && cfg->les != 1) || cfg->precision != CB_FP64 || (cfg->les && cfg->calc_sigma) || cfg->flux != 0 ||
      cfg->weno_order != 3)
    return na_fail(CB_E_UNSUPPORTED, "option combination not built");
  if (cfg->visT && !(cfg->tref > 0.0)) return na_fail(CB_E_ARG, "Tref must be > 0 with visT");
  DevCfg d{};
  d.mx = cfg->mx; d.my = cfg->my; d.mz = cfg->mz;
  d.px = ((cfg->mx + 4 + 15) / 16) * 16;
  d.py = cfg->my + 4;
  d.pz = cfg->mz + 4;
  d.plane = (long long)d.px * d.py * d.pz;
  if (d.plane > CB_NOALLOC_MAX_PLANE) {
    char buf[200];
    snprintf(buf, sizeof(buf), "grid %dx%dx%d needs %lld padded nodes per field, above the limit %lld (CB_NOALLOC_MAX_PLANE)",
             cfg->mx, cfg->my, cfg->mz, d.plane, (long long)CB_NOALLOC_MAX_PLANE);
    return na_fail(CB_E_ARG, buf);
  }
  for (int b = 0; b < 6; b++) d.bctype[b] = cfg->bctype[b];
  d.les = cfg->les; d.inviscid = cfg->inviscid; d.fluxorder = cfg->fluxorder; d.eno_order = cfg->eno_order;
  d.central = cfg->central; d.isothermal = cfg->isothermal;
  d.s_x = cfg->s_x; d.s_y = cfg->s_y; d.s_z = cfg->s_z;
  d.ren = cfg->ren; d.ma = cfg->ma; d.pr = cfg->pr; d.gamma = cfg->gamma; d.dt = cfg->dt; d.st = cfg->st;
  d.cs_const = cfg->cs_const; d.ci = cfg->ci; d.ratio = cfg->ratio;
  d.inv_ren = 1. / cfg->ren;
  d.inv_ren_half = 1. / cfg->ren * 0.5;
  set_sutherland(d, cfg->visT, cfg->tref, cfg->ren, cfg->gamma, cfg->ma);
  d.twod = cfg->twod;  // -twoD 1: no i-face fluxes
  d.gm1 = cfg->gamma - 1.0;
  d.kheat = cfg->gamma / cfg->pr / (cfg->gamma - 1.0);
  d.nvq = 0;  // nvert is a caller-owned device array: read it from global memory
  d.flux = 0;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return na_fail(CB_E_CUDA, "no current CUDA device");
  NaDevice &nd = g_dev[dev];
  {
    // device addresses of the arrays on the current device, every call: a
    // device reset since the last call would have moved them
    double *scratch = nullptr, **ptab = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&scratch, na_scratch);
    if (e != cudaSuccess) return na_fail(CB_E_CUDA, cudaGetErrorString(e));
    e = cudaGetSymbolAddress((void **)&ptab, na_ptab);
    if (e != cudaSuccess) return na_fail(CB_E_CUDA, cudaGetErrorString(e));
    if (!nd.ready || scratch != nd.scratch || ptab != nd.ptab) {
      // first call on this device (or the module was reloaded): the kernels'
      // shared-memory opt-in
      nd.ready = false;
      if ((e = na_attr<true, true>()) != cudaSuccess || (e = na_attr<true, false>()) != cudaSuccess ||
          (e = na_attr<false, true>()) != cudaSuccess || (e = na_attr<false, false>()) != cudaSuccess)
        return na_fail(CB_E_CUDA, cudaGetErrorString(e));
      nd.scratch = scratch;
      nd.ptab = ptab;
      nd.ready = true;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto grid_for = [&](long long work) {
    long long b = (work + 255) / 256, cap = (long long)sms * 8;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
  };

  const size_t P = (size_t)d.plane;
  NaPtrs tab{};
  for (int p = 0; p < NA_NPLANES; p++) tab.p[p] = nd.scratch + P * p;
  na_set_ptab<<<1, 32, 0, s>>>(tab);
  double **pt = nd.ptab;
  double *const *planes = (double *const *)pt;

  const long long nn = (long long)d.mx * d.my * d.mz;
  const long long all = (long long)(d.mx + 4) * (d.my + 4) * (d.mz + 4);
  // the RHS planes keep the last call's values: boundary nodes must read zero
  cudaMemsetAsync(tab.p[NA_RHS], 0, sizeof(double) * P * 5, s);
  // FormMetrics from the caller's coordinates
  unpack_kernel<<<grid_for(nn), 256, 0, s>>>(d, d_coor, 3, pt + NA_COOR);
  metrics_interior_kernel<<<grid_for(nn), 256, 0, s>>>(d, (const double *const *)(pt + NA_COOR), pt + NA_MET, tab.p[NA_AJ]);
  for (int f = 0; f < 6; f++) metrics_boundary_kernel<<<grid_for(nn / 4 + 1), 256, 0, s>>>(d, pt + NA_MET, tab.p[NA_AJ], f);
  ghost_fill_kernel<<<grid_for(all), 256, 0, s>>>(d, pt + NA_MET, 10);  // 9 metrics + aj are contiguous
  delta2_kernel<<<grid_for((long long)P), 256, 0, s>>>(d, tab.p[NA_AJ], tab.p[NA_DELTA2]);
  // state, mask and eddy viscosity into padded planes with their ghost layers
  unpack_kernel<<<grid_for(nn), 256, 0, s>>>(d, d_q, 5, pt + NA_Q);
  ghost_fill_kernel<<<grid_for(all), 256, 0, s>>>(d, pt + NA_Q, 5);
  unpack_kernel<<<grid_for(nn), 256, 0, s>>>(d, d_nvert, 1, pt + NA_NVERT);
  if (d_nut) {
    unpack_kernel<<<grid_for(nn), 256, 0, s>>>(d, d_nut, 1, pt + NA_NUT);
  } else {
    cudaMemsetAsync(tab.p[NA_NUT], 0, sizeof(double) * P, s);
  }
  ghost_fill_kernel<<<grid_for(all), 256, 0, s>>>(d, pt + NA_NVERT, 2);  // nvert and nu_t are contiguous

  DevFields F{};
  for (int q = 0; q < 5; q++) {
    F.q[q] = tab.p[NA_Q + q];
    F.qold[q] = tab.p[NA_Q + q];
    F.qout[q] = nullptr;
    F.rhs[q] = tab.p[NA_RHS + q];
  }
  for (int e = 0; e < 3; e++)
    for (int q = 0; q < 3; q++) F.met[e][q] = tab.p[NA_MET + 3 * e + q];
  F.aj = tab.p[NA_AJ];
  F.nvert = tab.p[NA_NVERT];
  F.nut = tab.p[NA_NUT];
  F.delta2 = tab.p[NA_DELTA2];
  F.status = nullptr;
  const int kchunk = d.mz - 2 < 16 ? d.mz - 2 : 16;
  const bool les = d.les != 0, visc = d.inviscid == 0;
  if (les && visc) na_launch_rhs<true, true>(d, F, kchunk, s);
  else if (les) na_launch_rhs<true, false>(d, F, kchunk, s);
  else if (visc) na_launch_rhs<false, true>(d, F, kchunk, s);
  else na_launch_rhs<false, false>(d, F, kchunk, s);
  pack_kernel<<<grid_for(nn), 256, 0, s>>>(d, (const double *const *)(pt + NA_RHS), 5, d_rhs);
  (void)planes;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(CB_E_CUDA, cudaGetErrorString(e));
  return CB_OK;
}
