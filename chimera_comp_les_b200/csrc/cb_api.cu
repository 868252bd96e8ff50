// C-ABI of libchimera_b200.so (declared in include/chimera_b200.h).
//
// One context = one block of the reference's DMDA resident on one GPU:
//   3 rotating state buffers (Q of the stage input, Q of the stage output and
//   Qold never collide, so no Q -> Qold copy is ever made), metrics, nvert and
//   nu_t, all as padded SoA planes in a single device allocation.
// A time step enqueues: [eddy viscosity + its ghost fill] then per RK stage
// [fused RHS/combine kernel, boundary + ghost fill kernel].  Steady-state
// steps replay CUDA graphs keyed by the buffer rotation.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/chimera_b200.h"
#include "cb_aux.cuh"
#include "cb_common.cuh"
#include "cb_dyn.cuh"
#include "cb_ibm.cuh"
#include "cb_ibm_host.h"
#include "cb_launch.h"
#include "cb_stage.cuh"

using namespace cb;

namespace {

constexpr int BX = SBX, BY = SBY;

struct GraphSlot {
  cudaGraphExec_t exec = nullptr;
};

}  // namespace

struct cb_ctx {
  cb_config cfg{};
  DevCfg dc{};
  int dev = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  double *arena = nullptr;
  size_t plane = 0;
  double *qb[3][5] = {};
  double *met[3][3] = {};
  double *aj = nullptr, *nvert = nullptr, *nut = nullptr, *delta2 = nullptr;
  double *rhsb[5] = {};
  // mixed form: FP32 metric vectors (with filter width and aj), FP64 metric divergence
  void *arena_mixed = nullptr;
  float4 *met4[3] = {};
  double *gcl[3] = {};
  float4 **ptab4 = nullptr;
  // shock sensor: final hybrid weights (a) and the pass buffer (b)
  double *sig_arena = nullptr;
  double *sig_a[3] = {}, *sig_b[3] = {};
  // dynamic Smagorinsky: velocity gradients (9), |S|, LM, MM, CS, lCS
  double *dyn_arena = nullptr;
  double dyn_tf_mult = 2.0;  // test-filter width over the filter width (les.c:598-601)
  bool have_refs = false;
  double *staging = nullptr;  // AoS upload/download buffer (5 doubles per node)
  // asynchronous host transfers (cb_upload_state_async / cb_download_state_async):
  // copy streams and two staging buffers per direction, allocated on first use
  cudaStream_t up_stream = nullptr, down_stream = nullptr;
  double *stg_in[2] = {}, *stg_out[2] = {};
  cudaEvent_t ev_in_copied[2] = {}, ev_in_free[2] = {}, ev_out_ready[2] = {}, ev_out_done[2] = {};
  int in_slot = 0, out_slot = 0;
  double **ptab = nullptr;    // device pointer tables
  unsigned *status = nullptr;
  bool fully_periodic = true;  // every face bctype 7: one fused periodic BC kernel
  bool nv0 = true;             // nvert is zero everywhere: the stage kernel's no-IBM variant
  bool nvz = true;             // nvert is zero everywhere (the eddy viscosity reads no nvert)
  int cur = 0;                // buffer with the current Q (== Qold between steps)
  int uc = -1;                // buffer of the last CalcUCat state, -1: none
  bool have_grid = false, have_state = false;
  int kchunk = 16;
  GraphSlot graphs[3][4][2];  // [cur][uc + 1][p_carry]
  bool use_graphs = true;
  // immersed bodies: interpolation after the stages, then FormBCS(user, 0)
  IbmBody ibm[CB_IBM_MAX_BODIES];
  double *ibm_arena = nullptr;  // 7 planes: spare (5) and psnap (1), the Q and P FormBCS reads, and pl
  double *spare = nullptr, *psnap = nullptr;
  double *coorxy = nullptr;  // node coordinates x, y (k-lo inflow codes 52 and 47), padded planes
  int *ti_dev = nullptr;     // step index user->ti on the device (code 47)
  double *pl = nullptr;  // the reference's P / lP after an immersed step
  bool p_carry = false;  // pl holds lP of the current state (no EqOfState since the interpolation)
  int ibm_twoD = 0, ibm_wallfunction = 0;
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, int>> ev_pairs_rhs, ev_pairs_other;
  double acc_rhs_ms = 0, acc_other_ms = 0;
  int acc_rhs_n = 0, acc_other_n = 0;
  std::string err;
};

static int fail(cb_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

#define CB_CUDA(ctx, call)                                                                  \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail(ctx, CB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

// device pointer tables inside ctx->ptab
enum { PT_Q0 = 0, PT_Q1 = 5, PT_Q2 = 10, PT_MET = 15, PT_COOR = 24, PT_RHS = 27, PT_NUT = 32, PT_MISC = 33, PT_GCL = 48,
       PT_SIGA = 56, PT_SIGB = 59, PT_PL = 64, PT_SNAP = 65, PT_DYN = 71, PT_N = 85 };
// PT_DYN + 0..8: du/dx .. dw/dz, 9: |S|, 10: LM, 11: MM, 12: CS, 13: lCS

// -les values that run the dynamic model: >= 2 except 10 (les.c:134-146
// single out 1 and 10; solvers.c:28 skips every model with 10)
static bool les_dynamic(const cb_config &f) { return f.les >= 2 && f.les != 10; }

static int grid_for(const cb_ctx *c, long long work, int block = 256) {
  long long b = (work + block - 1) / block;
  long long cap = (long long)c->sms * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

static DevFields fields_for(cb_ctx *c, int in, int old, int out) {
  DevFields F{};
  for (int q = 0; q < 5; q++) {
    F.q[q] = c->qb[in][q];
    F.qold[q] = c->qb[old][q];
    F.qout[q] = out >= 0 ? c->qb[out][q] : nullptr;
    F.rhs[q] = c->rhsb[q];
  }
  for (int e = 0; e < 3; e++)
    for (int q = 0; q < 3; q++) F.met[e][q] = c->met[e][q];
  F.aj = c->aj;
  F.nvert = c->nvert;
  F.nut = c->nut;
  F.delta2 = c->delta2;
  for (int e = 0; e < 3; e++) F.met4[e] = c->met4[e];
  for (int a = 0; a < 3; a++) F.sig[a] = c->sig_a[a];
  for (int a = 0; a < 3; a++) F.gcl[a] = c->gcl[a];
  F.status = c->status;
  F.cx = c->coorxy;
  F.cy = c->coorxy ? c->coorxy + c->plane : nullptr;
  F.ti = c->ti_dev;
  return F;
}

// Flux bits of the stage kernel: Roe, WENO5-JS, and with LES and the sensor
// off the constant blend weight s_x = s_y = s_z when it is exactly 1 or 0.
static int flux_bits(const cb_ctx *c) {
  int fl = (c->dc.flux == 1 ? FLUX_ROE : 0) | (c->cfg.weno_order == 5 ? FLUX_W5 : 0);
  const cb_config &f = c->cfg;
  if (f.les && !f.calc_sigma && f.s_x == f.s_y && f.s_y == f.s_z) {
    if (f.s_x == 1.0) fl |= FLUX_SIGMA1;
    else if (f.s_x == 0.0) fl |= FLUX_SIGMA0;
  }
  // every face periodic or an interface, no 2-D mode, MUSCL (or WENO5-JS,
  // whose reconstruction the W5 bit selects): the PLAIN variants
  bool per = f.twod == 0 && (f.fluxorder == 2 || f.weno_order == 5);
  for (int s = 0; s < 6; s++) per = per && f.bctype[s] == 7;
  if (per) fl |= FLUX_PLAIN;
  return fl;
}

static cudaError_t launch_stage(cb_ctx *c, const DevFields &F, int istage, double alfa, double beta, double adt, bool rhs_mode) {
  const bool les = c->cfg.les != 0, visc = c->cfg.inviscid == 0, mix = c->cfg.precision == CB_MIXED;
  return launch_stage_any(mix, les, c->dc, F, istage, alfa, beta, adt, c->kchunk, visc, rhs_mode, flux_bits(c),
                          c->nv0 && !rhs_mode, (mix ? 2 : 1) * c->sms, c->stream);
}

static cudaEvent_t ev_get(cb_ctx *c, int idx) {
  while ((int)c->ev_pool.size() <= idx) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->ev_pool.push_back(e);
  }
  return c->ev_pool[idx];
}

// timing helpers: record a pair of events around a launch
struct TimedScope {
  cb_ctx *c;
  bool rhs;
  int a = -1;
  TimedScope(cb_ctx *ctx, bool is_rhs) : c(ctx), rhs(is_rhs) {
    if (!c->timing) return;
    a = (int)(c->ev_pairs_rhs.size() + c->ev_pairs_other.size()) * 2;
    cudaEventRecord(ev_get(c, a), c->stream);
  }
  ~TimedScope() {
    if (!c->timing) return;
    cudaEventRecord(ev_get(c, a + 1), c->stream);
    (rhs ? c->ev_pairs_rhs : c->ev_pairs_other).push_back({a, a + 1});
  }
};

static void harvest_timing(cb_ctx *c) {
  if (c->ev_pairs_rhs.empty() && c->ev_pairs_other.empty()) return;
  cudaStreamSynchronize(c->stream);
  for (auto &p : c->ev_pairs_rhs) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev_pool[p.first], c->ev_pool[p.second]);
    c->acc_rhs_ms += ms;
    c->acc_rhs_n++;
  }
  for (auto &p : c->ev_pairs_other) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev_pool[p.first], c->ev_pool[p.second]);
    c->acc_other_ms += ms;
    c->acc_other_n++;
  }
  c->ev_pairs_rhs.clear();
  c->ev_pairs_other.clear();
}

// Hybrid weights of the shock sensor from the stage input `in` (istage 0 of
// formConvectionLES): three passes, each followed by the DMGlobalToLocal wrap.
// P: the pressure plane the first stage reads after an immersed step (lP
// carried from the interpolation), else null (the EOS of the input).
static int sigma_update(cb_ctx *c, int in, const double *P) {
  if (!c->dc.calc_sigma) return CB_OK;
  TimedScope ts(c, false);
  const int g = grid_for(c, (long long)c->plane);
  const long long sh = shell_count(c->dc);
  sigma_sensor_kernel<<<g, 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + 5 * in), c->ptab + PT_SIGA, P);
  ghost_fill_kernel<<<grid_for(c, sh), 256, 0, c->stream>>>(c->dc, c->ptab + PT_SIGA, 3);
  sigma_filter_kernel<<<g, 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + PT_SIGA), c->ptab + PT_SIGB);
  ghost_fill_kernel<<<grid_for(c, sh), 256, 0, c->stream>>>(c->dc, c->ptab + PT_SIGB, 3);
  sigma_post_kernel<<<g, 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + PT_SIGB), c->ptab + PT_SIGA);
  ghost_fill_kernel<<<grid_for(c, sh), 256, 0, c->stream>>>(c->dc, c->ptab + PT_SIGA, 3);
  CB_CUDA(c, cudaGetLastError());
  return CB_OK;
}

// Compute_Smagorinsky_Constant_1 with -les 2 (les.c:151-1472) into the CS
// plane, from the current state and the recorded CalcUCat state.
static int dynamic_cs(cb_ctx *c) {
  TimedScope ts(c, false);
  const double *const *q = (const double *const *)(c->ptab + 5 * c->cur);
  const double *const *qu = c->uc >= 0 ? (const double *const *)(c->ptab + 5 * c->uc) : nullptr;
  double *base = c->dyn_arena;
  const size_t pl = c->plane;
  const DynPlanes P{c->ptab + PT_DYN, base + 9 * pl, base + 10 * pl, base + 11 * pl, base + 12 * pl, base + 13 * pl};
  const cb_config &f = c->cfg;
  const DynOpts o{f.les, f.max_cs, c->dyn_tf_mult, f.i_homo_filter, f.j_homo_filter, f.k_homo_filter};
  CB_CUDA(c, dyn_cs_enqueue(c->dc, o, q, qu, (const double *const *)(c->ptab + PT_MET), c->aj, c->nvert, P, c->sms,
                            c->stream));
  return CB_OK;
}

static int nut_update(cb_ctx *c) {
  // Compute_eddy_viscosity_LES from the recorded state (or zero velocity).
  const long long work = (long long)(c->dc.mx - 2) * (c->dc.my - 2) * (c->dc.mz - 2);
  const bool dyn = les_dynamic(c->cfg);
  if (c->cfg.les == 10) {  // Cs = 0 (les.c:134-137): nu_t stays zero
    CB_CUDA(c, cudaMemsetAsync(c->nut, 0, sizeof(double) * c->plane, c->stream));
    return CB_OK;
  }
  if (dyn) {
    int e = dynamic_cs(c);
    if (e) return e;
  }
  {
    TimedScope ts(c, false);
    const double *const *qu = c->uc >= 0 ? (const double *const *)(c->ptab + 5 * c->uc) : nullptr;
    if (c->cfg.precision == CB_MIXED && !dyn) {  // the mixed form's SGS terms run in FP32
      CB_CUDA(c, launch_eddy_mixed(c->dc, qu, c->met4, c->nvz ? nullptr : c->nvert, c->nut, c->sms, c->stream));
    } else {
      const int ekc = eddy_kchunk(c->dc, c->sms);
      eddy_viscosity_kernel<<<eddy_grid(c->dc, ekc), dim3(EDDY_BX, EDDY_BY), 0, c->stream>>>(
          c->dc, qu, (const double *const *)(c->ptab + PT_MET), c->aj, c->delta2, c->nvz ? nullptr : c->nvert, c->nut,
          ekc, dyn ? (const double *const *)(c->ptab + 5 * c->cur) : nullptr,
          dyn ? c->dyn_arena + 12 * c->plane : nullptr);
    }
  }
  {
    TimedScope ts(c, false);
    ghost_fill_kernel<<<grid_for(c, shell_count(c->dc)), 256, 0, c->stream>>>(c->dc, c->ptab + PT_NUT, 1);
  }
  CB_CUDA(c, cudaGetLastError());
  return CB_OK;
}

static void rk_coeffs(const cb_ctx *c, int s, double *alfa, double *beta) {
  double a[3] = {1., 1 / 4., 2 / 3.}, b[3] = {1., 3 / 4., 1 / 3.};  // solvers.c:233-234
  if (c->cfg.fluxorder < 3) { a[1] = 1 / 2.; b[1] = 1 / 2.; }       // solvers.c:239-241
  *alfa = a[s];
  *beta = b[s];
}

static bool ibm_active(const cb_ctx *c) {
  for (const auto &b : c->ibm)
    if (b.n > 0) return true;
  return false;
}

// Five sweeps of ibm_interpolation_advanced for one body on the current state.
// rho_old: the density plane of Qold, which -isothermal 2 reads.
static int ibm_sweeps(cb_ctx *c, const IbmBody &b, int add_dundt, const double *rho_old) {
  const IbmDev d = b.dev();
  const int g = grid_for(c, b.n);
  const int slip = (c->cfg.inviscid || c->ibm_wallfunction == 3) ? 1 : 0;  // ibm_iso.c:2721
  const int iso1 = c->cfg.isothermal == 1 ? 1 : 0;
  const int wf2 = c->ibm_wallfunction == 2 ? 1 : 0;
  const bool iso2 = c->cfg.isothermal == 2;
  const double a_sound = sqrt(c->cfg.twall / (c->cfg.ma * c->cfg.ma));  // ibm_iso.c:2768, the host's sqrt
  for (int s = 0; s < IBM_SWEEPS; s++) {
    ibm_interp_kernel<<<g, 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + 5 * c->cur), c->pl, d,
                                                add_dundt, c->ibm_twoD, slip, iso1, wf2, iso2 ? rho_old : nullptr,
                                                a_sound);
    if (iso2) {
      ibm_iso2_chain_kernel<<<1, IBM_CHAIN_NT, 0, c->stream>>>(c->dc, d, s == 0 ? 1 : 0, a_sound);
      ibm_iso2_finish_kernel<<<g, 256, 0, c->stream>>>(c->dc, d, add_dundt);
    }
    ibm_scatter_kernel<<<g, 256, 0, c->stream>>>(c->dc, c->ptab + 5 * c->cur, c->pl, d);
  }
  CB_CUDA(c, cudaGetLastError());
  return CB_OK;
}

// EqOfState of the current state into the pressure plane (solvers.c:279).
static int eos_to_plane(cb_ctx *c) {
  eos_plane_kernel<<<grid_for(c, (long long)c->plane), 256, 0, c->stream>>>(
      c->dc, (const double *const *)(c->ptab + 5 * c->cur), c->pl);
  CB_CUDA(c, cudaGetLastError());
  return CB_OK;
}

// FormBCS(user, 0) after the interpolation (solvers.c:286): the boundary of
// the current state from a snapshot of it and of the pressure plane (the
// reference's lQ and lP), Qold from buffer `old`; the periodic copies move P
// with Q; then the ghost wrap of both that FormBCS ends with
// (rhs.c:1305-1308).  No EqOfState follows: the pressure plane is carried.
static int formbcs_zero(cb_ctx *c, int old) {
  // snapshot of Q and P within five layers of the faces: FormBCS reads its lQ / lP
  // at most two nodes beyond the boundary layer, on either side
  if (std::min(c->dc.mx, std::min(c->dc.my, c->dc.mz)) >= 6) {
    const long long thick = thick_shell_count(c->dc, 5);
    thick_shell_copy_kernel<<<grid_for(c, thick), 256, 0, c->stream>>>(
        c->dc, 5, (const double *const *)(c->ptab + 5 * c->cur), c->ptab + PT_SNAP, 5);
    thick_shell_copy_kernel<<<grid_for(c, thick), 256, 0, c->stream>>>(
        c->dc, 5, (const double *const *)(c->ptab + PT_PL), c->ptab + PT_SNAP + 5, 1);
  } else {  // every node lies within five layers of a face
    CB_CUDA(c, cudaMemcpyAsync(c->spare, c->qb[c->cur][0], sizeof(double) * 5 * c->plane, cudaMemcpyDeviceToDevice,
                               c->stream));
    CB_CUDA(c, cudaMemcpyAsync(c->psnap, c->pl, sizeof(double) * c->plane, cudaMemcpyDeviceToDevice, c->stream));
  }
  DevFields F = fields_for(c, c->cur, old, c->cur);
  for (int q = 0; q < 5; q++) F.q[q] = c->spare + c->plane * q;
  F.pin = c->psnap;
  const long long shell = shell_count(c->dc);
  if (c->fully_periodic) {
    bc_periodic_kernel<<<grid_for(c, shell), 256, 0, c->stream>>>(c->dc, F);
    bc_periodic_p_kernel<<<grid_for(c, shell), 256, 0, c->stream>>>(c->dc, c->psnap, c->pl);
  } else {
    const long long face = (long long)std::max(c->dc.mx, c->dc.my) * std::max(c->dc.my, c->dc.mz);
    for (int dir = 0; dir < 3; dir++) bc_face_kernel<<<grid_for(c, face), 256, 0, c->stream>>>(c->dc, F, dir, 0.0);
    for (int dir = 0; dir < 3; dir++)
      if (c->dc.bctype[2 * dir] == 7) {
        bc_periodic_dir_kernel<<<grid_for(c, face), 256, 0, c->stream>>>(c->dc, F, dir);
        bc_periodic_dir_p_kernel<<<grid_for(c, face), 256, 0, c->stream>>>(c->dc, c->psnap, c->pl, dir);
      }
    ghost_fill_kernel<<<grid_for(c, shell), 256, 0, c->stream>>>(c->dc, c->ptab + 5 * c->cur, 5);
    ghost_fill_kernel<<<grid_for(c, shell), 256, 0, c->stream>>>(c->dc, c->ptab + PT_PL, 1);
  }
  CB_CUDA(c, cudaGetLastError());
  return CB_OK;
}

// Enqueue one time step (no graph).
static int enqueue_step(cb_ctx *c) {
  if (c->dc.bctype[4] == 47) step_index_advance_kernel<<<1, 1, 0, c->stream>>>(c->ti_dev);
  if (c->cfg.les && c->cfg.les != 10 && !c->cfg.inviscid) {  // solvers.c:28
    int e = nut_update(c);
    if (e) return e;
  }
  const int ns = c->cfg.fluxorder;
  const int old = c->cur;
  const int A = (c->cur + 1) % 3, B = (c->cur + 2) % 3;
  int in = c->cur;
  const long long shell = shell_count(c->dc);
  for (int s = 0; s < ns; s++) {
    const int out = (s % 2 == 0) ? A : B;
    double alfa, beta;
    rk_coeffs(c, s, &alfa, &beta);
    const double adt = alfa * c->cfg.dt * c->cfg.st;
    DevFields F = fields_for(c, in, old, out);
    if (s == 0 && c->p_carry) F.pin = c->pl;  // lP carried from the interpolation of the previous step
    if (s == 0) {
      int e = sigma_update(c, in, c->p_carry ? c->pl : nullptr);
      if (e) return e;
    }
    {
      TimedScope ts(c, true);
      CB_CUDA(c, launch_stage(c, F, s, alfa, beta, adt, false));
    }
    {
      TimedScope ts(c, false);
      if (c->fully_periodic) {
        bc_periodic_kernel<<<grid_for(c, shell), 256, 0, c->stream>>>(c->dc, F);
      } else {  // FormBCS with boundary codes (rhs.c:477-1227)
        bc_combine_kernel<<<grid_for(c, shell), 256, 0, c->stream>>>(c->dc, F, s, alfa, beta, adt);
        const long long face = (long long)std::max(c->dc.mx, c->dc.my) * std::max(c->dc.my, c->dc.mz);
        for (int dir = 0; dir < 3; dir++)
          bc_face_kernel<<<grid_for(c, face), 256, 0, c->stream>>>(c->dc, F, dir, alfa);
        for (int dir = 0; dir < 3; dir++)
          if (c->dc.bctype[2 * dir] == 7)
            bc_periodic_dir_kernel<<<grid_for(c, face), 256, 0, c->stream>>>(c->dc, F, dir);
        ghost_fill_kernel<<<grid_for(c, shell), 256, 0, c->stream>>>(c->dc, c->ptab + 5 * out, 5);
      }
    }
    CB_CUDA(c, cudaGetLastError());
    if (!c->cfg.inviscid) c->uc = in;  // CalcUCat inside formRHS keeps the stage input
    in = out;
  }
  c->cur = in;
  c->p_carry = false;
  if (ibm_active(c)) {  // solvers.c:279-288
    TimedScope ts(c, false);
    int e = eos_to_plane(c);
    if (e) return e;
    for (const auto &b : c->ibm)
      if (b.n > 0) {
        e = ibm_sweeps(c, b, 1, c->qb[old][0]);  // Qold: the step's input, untouched by its stages
        if (e) return e;
      }
    e = formbcs_zero(c, old);
    if (e) return e;
    c->p_carry = true;
  }
  return CB_OK;
}

static int fill_ptab(cb_ctx *c) {
  double *h[PT_N] = {};
  for (int b = 0; b < 3; b++)
    for (int q = 0; q < 5; q++) h[5 * b + q] = c->qb[b][q];
  for (int e = 0; e < 3; e++)
    for (int q = 0; q < 3; q++) h[PT_MET + 3 * e + q] = c->met[e][q];
  for (int q = 0; q < 5; q++) h[PT_RHS + q] = c->rhsb[q];
  h[PT_NUT] = c->nut;
  h[PT_MISC + 0] = c->aj;
  h[PT_MISC + 1] = c->nvert;
  for (int e = 0; e < 3; e++)
    for (int q = 0; q < 3; q++) h[PT_MISC + 2 + 3 * e + q] = c->met[e][q];
  h[PT_MISC + 11] = c->aj;
  for (int a = 0; a < 3; a++) h[PT_GCL + a] = c->gcl[a];
  for (int a = 0; a < 3; a++) { h[PT_SIGA + a] = c->sig_a[a]; h[PT_SIGB + a] = c->sig_b[a]; }
  h[PT_PL] = c->pl;
  for (int q = 0; q < 5; q++) h[PT_SNAP + q] = c->spare ? c->spare + c->plane * q : nullptr;
  h[PT_SNAP + 5] = c->psnap;
  for (int a = 0; a < 14; a++) h[PT_DYN + a] = c->dyn_arena ? c->dyn_arena + c->plane * a : nullptr;
  CB_CUDA(c, cudaMemcpyAsync(c->ptab, h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  if (c->ptab4) CB_CUDA(c, cudaMemcpyAsync(c->ptab4, c->met4, sizeof(c->met4), cudaMemcpyHostToDevice, c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

static void invalidate_graphs(cb_ctx *c) {
  for (auto &row : c->graphs)
    for (auto &col : row)
      for (auto &g : col)
        if (g.exec) { cudaGraphExecDestroy(g.exec); g.exec = nullptr; }
}

extern "C" {

int cb_abi_version(void) { return CB_ABI_VERSION; }

int cb_set_time_index(cb_ctx *c, int ti) {
  if (!c) return CB_E_ARG;
  CB_CUDA(c, cudaMemcpyAsync(c->ti_dev, &ti, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

void cb_config_default(cb_config *cfg, int mx, int my, int mz) {
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->mx = mx; cfg->my = my; cfg->mz = mz;
  for (int b = 0; b < 6; b++) cfg->bctype[b] = 7;
  cfg->les = 0; cfg->inviscid = 0; cfg->fluxorder = 3; cfg->eno_order = 2; cfg->central = 2; cfg->isothermal = 0;
  cfg->s_x = cfg->s_y = cfg->s_z = 1.0;
  cfg->ren = 3000.; cfg->ma = 2.81; cfg->pr = 0.72; cfg->gamma = 1.4; cfg->dt = 0.01; cfg->st = 1.;
  cfg->cs_const = 0.03; cfg->ci = 0.06; cfg->ratio = 0.;
  cfg->precision = CB_FP64;
  cfg->device = 0;
  cfg->calc_sigma = 0;
  cfg->s_x_min = cfg->s_y_min = cfg->s_z_min = 0.;
  cfg->sigma_thrsh = 0.00001;  // rhs.c:3322
  cfg->max_cs = 0.05;          // les.c:151
  cfg->twall = 1.;             // rhs.c:486
  cfg->twod = 0;
  cfg->visT = 0;
  cfg->tref = 273.15;          // rhs.c:1410
  cfg->abc = 0;
  cfg->weno_order = 3;         // the reference's WENO3
}

int cb_create(const cb_config *cfg, cb_ctx **out) {
  if (!cfg || !out) return CB_E_ARG;
  *out = nullptr;
  cb_ctx *c = new cb_ctx();
  c->cfg = *cfg;
  auto bail = [&](int code, const char *msg) {
    fprintf(stderr, "chimera_b200: cb_create: %s\n", msg);
    cb_destroy(c);
    return code;
  };
  if (cfg->mx < 5 || cfg->my < 5 || cfg->mz < 5) return bail(CB_E_ARG, "grid must have at least 5 nodes per direction");
  {
    const int *bc = cfg->bctype;
    for (int d = 0; d < 3; d++)
      if ((bc[2 * d] == 7) != (bc[2 * d + 1] == 7))
        return bail(CB_E_UNSUPPORTED, "a periodic direction needs bctype 7 on both faces");
    c->fully_periodic = true;
    for (int b = 0; b < 6; b++) c->fully_periodic = c->fully_periodic && bc[b] == 7;
  }
  if (cfg->fluxorder < 1 || cfg->fluxorder > 3) return bail(CB_E_ARG, "fluxorder must be 1, 2 or 3");
  if (cfg->weno_order != 3 && cfg->weno_order != 5) return bail(CB_E_ARG, "weno_order must be 3 or 5");
  if (cfg->weno_order == 5 && cfg->fluxorder != 3) return bail(CB_E_ARG, "weno_order 5 needs fluxorder 3");
  if (cfg->eno_order != 2 && cfg->eno_order != 3) return bail(CB_E_ARG, "ENOorder must be 2 or 3");
  if (cfg->les < 0) return bail(CB_E_ARG, "les must be >= 0");
  if (les_dynamic(*cfg) && !(cfg->max_cs >= 0.0)) return bail(CB_E_ARG, "max_cs must be >= 0");
  if (cfg->visT && !(cfg->tref > 0.0)) return bail(CB_E_ARG, "Tref must be > 0 with visT");
  c->nv0 = !cfg->visT;  // nvert starts zero; the no-IBM variants carry no Sutherland law
  if (cfg->precision != CB_FP64 && cfg->precision != CB_MIXED) return bail(CB_E_ARG, "precision must be CB_FP64 or CB_MIXED");
  if (cfg->flux != 0 && cfg->flux != 1) return bail(CB_E_ARG, "flux must be 0 (Rusanov) or 1 (Roe)");
  c->dev = cfg->device;
  if (cudaSetDevice(c->dev) != cudaSuccess) return bail(CB_E_CUDA, "cudaSetDevice failed");
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->dev);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(CB_E_CUDA, "stream");
  if (stage_attrs_all(cfg->precision == CB_MIXED) != cudaSuccess)
    return bail(CB_E_CUDA, "stage kernel shared-memory opt-in failed");
  DevCfg &d = c->dc;
  d.mx = cfg->mx; d.my = cfg->my; d.mz = cfg->mz;
  d.px = ((cfg->mx + 4 + 15) / 16) * 16;
  d.py = cfg->my + 4;
  d.pz = cfg->mz + 4;
  d.plane = (long long)d.px * d.py * d.pz;
  for (int b = 0; b < 6; b++) d.bctype[b] = cfg->bctype[b];
  d.les = cfg->les; d.inviscid = cfg->inviscid; d.fluxorder = cfg->fluxorder; d.eno_order = cfg->eno_order;
  d.central = cfg->central; d.isothermal = cfg->isothermal;
  d.s_x = cfg->s_x; d.s_y = cfg->s_y; d.s_z = cfg->s_z;
  d.ren = cfg->ren; d.ma = cfg->ma; d.pr = cfg->pr; d.gamma = cfg->gamma; d.dt = cfg->dt; d.st = cfg->st;
  d.cs_const = cfg->cs_const; d.ci = cfg->ci; d.ratio = cfg->ratio;
  d.inv_ren = 1. / cfg->ren;
  d.inv_ren_half = 1. / cfg->ren * 0.5;
  set_sutherland(d, cfg->visT, cfg->tref, cfg->ren, cfg->gamma, cfg->ma);
  d.gm1 = cfg->gamma - 1.0;
  d.kheat = cfg->gamma / cfg->pr / (cfg->gamma - 1.0);
  d.nvq = 1;  // nvert starts zero
  if ((long long)(cfg->mx + 4) * (cfg->my + 4) * (cfg->mz + 4) >= (1LL << 31))
    return bail(CB_E_ARG, "grid too large for 32-bit boundary indexing");
  d.calc_sigma = (cfg->les && cfg->calc_sigma) ? 1 : 0;
  d.s_x_min = cfg->s_x_min; d.s_y_min = cfg->s_y_min; d.s_z_min = cfg->s_z_min;
  d.ks = cfg->sigma_thrsh;
  d.flux = cfg->flux;
  d.twall = cfg->twall;
  d.twod = cfg->twod;
  d.abc = cfg->abc;
  c->plane = (size_t)d.plane;
  // planes: 15 state + 9 metrics + aj + nvert + nut + LES filter width = 28
  const int nplanes = 28;
  const size_t bytes = sizeof(double) * c->plane * nplanes;
  if (cudaMalloc(&c->arena, bytes) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc arena");
  if (cudaMemsetAsync(c->arena, 0, bytes, c->stream) != cudaSuccess) return bail(CB_E_CUDA, "memset");
  int p = 0;
  for (int b = 0; b < 3; b++)
    for (int q = 0; q < 5; q++) c->qb[b][q] = c->arena + c->plane * (p++);
  for (int e = 0; e < 3; e++)
    for (int q = 0; q < 3; q++) c->met[e][q] = c->arena + c->plane * (p++);
  c->aj = c->arena + c->plane * (p++);
  c->nvert = c->arena + c->plane * (p++);
  c->nut = c->arena + c->plane * (p++);
  c->delta2 = c->arena + c->plane * (p++);
  const size_t nn = (size_t)cfg->mx * cfg->my * cfg->mz;
  if (cudaMalloc(&c->staging, sizeof(double) * 5 * nn) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc staging");
  if (cfg->precision == CB_MIXED) {
    const size_t mbytes = sizeof(float4) * c->plane * 3 + sizeof(double) * c->plane * 3;
    if (cudaMalloc(&c->arena_mixed, mbytes) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc mixed planes");
    if (cudaMemsetAsync(c->arena_mixed, 0, mbytes, c->stream) != cudaSuccess) return bail(CB_E_CUDA, "memset");
    float4 *f = (float4 *)c->arena_mixed;
    for (int e = 0; e < 3; e++) c->met4[e] = f + c->plane * e;
    double *g = (double *)(f + c->plane * 3);
    for (int a = 0; a < 3; a++) c->gcl[a] = g + c->plane * a;
    if (cudaMalloc(&c->ptab4, sizeof(float4 *) * 3) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc ptab4");
  }
  if (les_dynamic(*cfg)) {
    c->dyn_tf_mult = cfg->testfilter_ik ? pow(5.0, 1. / 3.) : 2.0;  // the host's pow, as the reference's
    if (cudaFuncSetAttribute(dyn_lm_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DYN_LM_SMEM) !=
        cudaSuccess)
      return bail(CB_E_CUDA, "dynamic-model kernel attributes");
    const size_t db = sizeof(double) * c->plane * 14;
    if (cudaMalloc(&c->dyn_arena, db) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc dynamic-model planes");
    if (cudaMemsetAsync(c->dyn_arena, 0, db, c->stream) != cudaSuccess) return bail(CB_E_CUDA, "memset");
  }
  if (c->dc.calc_sigma) {
    const size_t sb = sizeof(double) * c->plane * 6;
    if (cudaMalloc(&c->sig_arena, sb) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc sensor planes");
    if (cudaMemsetAsync(c->sig_arena, 0, sb, c->stream) != cudaSuccess) return bail(CB_E_CUDA, "memset");
    for (int a = 0; a < 3; a++) {
      c->sig_a[a] = c->sig_arena + c->plane * a;
      c->sig_b[a] = c->sig_arena + c->plane * (3 + a);
    }
  }
  if (cudaMalloc(&c->ptab, sizeof(double *) * PT_N) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc ptab");
  if (cudaMalloc(&c->status, sizeof(unsigned)) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc status");
  if (cudaMalloc(&c->ti_dev, sizeof(int)) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc step index");
  cudaMemsetAsync(c->ti_dev, 0, sizeof(int), c->stream);
  if (cfg->bctype[4] == 52 || cfg->bctype[4] == 47) {  // the inflow codes read the node coordinates
    if (cudaMalloc(&c->coorxy, sizeof(double) * c->plane * 2) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc coordinates");
    cudaMemsetAsync(c->coorxy, 0, sizeof(double) * c->plane * 2, c->stream);
  }
  cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->stream);
  if (fill_ptab(c)) return bail(CB_E_CUDA, "pointer table");
  // k-chunk: whole waves of the resident blocks (1 per SM in the FP64 form,
  // 2 in the mixed form); a chunk's prologue costs about one plane.  The
  // autotuner (cb_autotune) refines this by measurement.
  {
    const int by = cfg->weno_order == 5 ? SBY_W5 : BY;
    const int tiles = ((cfg->mx - 2 + BX - 1) / BX) * ((cfg->my - 2 + by - 1) / by);
    const int nk = cfg->mz - 2;
    const int slots = c->sms * (cfg->precision == CB_MIXED ? 2 : 1);
    double best = 1e30;
    for (int kc = 4; kc <= nk; kc++) {
      const int chunks = (nk + kc - 1) / kc;
      const long long blocks = (long long)tiles * chunks;
      const long long waves = (blocks + slots - 1) / slots;
      const double cost = (double)waves * (kc + 1.0);
      if (cost < best) { best = cost; c->kchunk = kc; }
    }
  }
  *out = c;
  return CB_OK;
}

void cb_destroy(cb_ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  invalidate_graphs(c);
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->rhsb[0]) cudaFree(c->rhsb[0]);
  if (c->arena) cudaFree(c->arena);
  if (c->staging) cudaFree(c->staging);
  if (c->up_stream) cudaStreamSynchronize(c->up_stream);
  if (c->down_stream) cudaStreamSynchronize(c->down_stream);
  for (int i = 0; i < 2; i++) {
    if (c->stg_in[i]) cudaFree(c->stg_in[i]);
    if (c->stg_out[i]) cudaFree(c->stg_out[i]);
    for (cudaEvent_t e : {c->ev_in_copied[i], c->ev_in_free[i], c->ev_out_ready[i], c->ev_out_done[i]})
      if (e) cudaEventDestroy(e);
  }
  if (c->up_stream) cudaStreamDestroy(c->up_stream);
  if (c->down_stream) cudaStreamDestroy(c->down_stream);
  if (c->arena_mixed) cudaFree(c->arena_mixed);
  if (c->ptab4) cudaFree(c->ptab4);
  if (c->sig_arena) cudaFree(c->sig_arena);
  if (c->dyn_arena) cudaFree(c->dyn_arena);
  for (auto &b : c->ibm) {
    if (b.surf) cudaFree(b.surf);
    if (b.list) cudaFree(b.list);
  }
  if (c->ibm_arena) cudaFree(c->ibm_arena);
  if (c->ptab) cudaFree(c->ptab);
  if (c->status) cudaFree(c->status);
  if (c->ti_dev) cudaFree(c->ti_dev);
  if (c->coorxy) cudaFree(c->coorxy);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char *cb_last_error(const cb_ctx *c) { return c ? c->err.c_str() : "null context"; }
void *cb_stream(cb_ctx *c) { return c ? (void *)c->stream : nullptr; }
long long cb_interior_nodes(const cb_ctx *c) {
  return c ? (long long)(c->cfg.mx - 2) * (c->cfg.my - 2) * (c->cfg.mz - 2) : 0;
}
int cb_stages(const cb_ctx *c) { return c ? c->cfg.fluxorder : 0; }
int cb_launches_per_step(const cb_ctx *c) {
  if (!c) return 0;
  int per_stage = 2;
  if (!c->fully_periodic) {
    per_stage = 1 + 1 + 3 + 1;
    for (int d = 0; d < 3; d++) per_stage += c->cfg.bctype[2 * d] == 7;
  }
  int ib = 0;
  if (ibm_active(c)) {
    ib += 1;  // EqOfState into the pressure plane
    for (const auto &b : c->ibm) ib += b.n > 0 ? 2 * IBM_SWEEPS : 0;
    // FormBCS(user, 0): no stage kernel, no RK combine; P copies and ghost wrap beside Q's
    int nper = 0;
    for (int d = 0; d < 3; d++) nper += c->cfg.bctype[2 * d] == 7;
    if (std::min(c->dc.mx, std::min(c->dc.my, c->dc.mz)) >= 6) ib += 2;  // the snapshots of Q and P near the faces
    ib += c->fully_periodic ? 2 : per_stage - 2 + nper + 1;
  }
  const cb_config &f = c->cfg;
  const bool homo = f.i_homo_filter || f.j_homo_filter || f.k_homo_filter;
  const bool box = f.i_homo_filter && f.j_homo_filter && f.k_homo_filter;
  int dyn = 0;  // the dynamic model's kernels
  if (les_dynamic(f) && !f.inviscid) {
    dyn = (homo || f.les == 3) ? 6 : 9;
    if (homo) dyn += 1 + (box ? 2 : (f.i_homo_filter ? 1 : 0));
  }
  const bool model = f.les && f.les != 10 && !f.inviscid;
  return (model ? 2 : 0) + dyn + per_stage * c->cfg.fluxorder + (c->dc.calc_sigma ? 6 : 0) + ib;
}

static int upload_planes(cb_ctx *c, const double *host, int nc, int pt_first, bool pinned_hint) {
  (void)pinned_hint;
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  CB_CUDA(c, cudaMemcpyAsync(c->staging, host, sizeof(double) * nc * nn, cudaMemcpyHostToDevice, c->stream));
  unpack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, c->staging, nc, c->ptab + pt_first);
  CB_CUDA(c, cudaGetLastError());
  const long long all = (long long)(c->dc.mx + 4) * (c->dc.my + 4) * (c->dc.mz + 4);
  ghost_fill_kernel<<<grid_for(c, all), 256, 0, c->stream>>>(c->dc, c->ptab + pt_first, nc);
  CB_CUDA(c, cudaGetLastError());
  return CB_OK;
}

int cb_set_grid(cb_ctx *c, const double *coor) {
  if (!c || !coor) return CB_E_ARG;
  // coordinates go into state buffer 2 temporarily (overwritten by uploads/steps)
  double *X[3] = {c->qb[2][0], c->qb[2][1], c->qb[2][2]};
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  CB_CUDA(c, cudaMemcpyAsync(c->staging, coor, sizeof(double) * 3 * nn, cudaMemcpyHostToDevice, c->stream));
  unpack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, c->staging, 3, c->ptab + PT_Q2);
  const long long work = (long long)nn;
  metrics_interior_kernel<<<grid_for(c, work), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + PT_Q2),
                                                                      c->ptab + PT_MET, c->aj);
  for (int f = 0; f < 6; f++)
    metrics_boundary_kernel<<<grid_for(c, work / 4 + 1), 256, 0, c->stream>>>(c->dc, c->ptab + PT_MET, c->aj, f);
  const long long all = (long long)(c->dc.mx + 4) * (c->dc.my + 4) * (c->dc.mz + 4);
  ghost_fill_kernel<<<grid_for(c, all), 256, 0, c->stream>>>(c->dc, c->ptab + PT_MISC + 2, 10);
  delta2_kernel<<<grid_for(c, all), 256, 0, c->stream>>>(c->dc, c->aj, c->delta2);
  CB_CUDA(c, cudaGetLastError());
  if (c->cfg.precision == CB_MIXED)
    CB_CUDA(c, launch_mixed_prep(c->dc, (const double *const *)(c->ptab + PT_MET), c->delta2, c->aj, c->ptab4,
                                 c->ptab + PT_GCL, grid_for(c, (long long)c->plane), c->stream));
  if (c->coorxy)  // x and y kept for the inflow codes that read them
    for (int q = 0; q < 2; q++)
      CB_CUDA(c, cudaMemcpyAsync(c->coorxy + c->plane * q, X[q], sizeof(double) * c->plane, cudaMemcpyDeviceToDevice,
                                 c->stream));
  // scrub buffer 2 (coordinates) so later ghost reads see zeros until written
  for (int q = 0; q < 3; q++) CB_CUDA(c, cudaMemsetAsync(X[q], 0, sizeof(double) * c->plane, c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->have_grid = true;
  invalidate_graphs(c);
  return CB_OK;
}

int cb_set_metrics(cb_ctx *c, const double *csi, const double *eta, const double *zet, const double *aj) {
  if (!c || !csi || !eta || !zet || !aj) return CB_E_ARG;
  int e;
  if ((e = upload_planes(c, csi, 3, PT_MET + 0, false))) return e;
  if ((e = upload_planes(c, eta, 3, PT_MET + 3, false))) return e;
  if ((e = upload_planes(c, zet, 3, PT_MET + 6, false))) return e;
  if ((e = upload_planes(c, aj, 1, PT_MISC + 0, false))) return e;
  const long long all = (long long)(c->dc.mx + 4) * (c->dc.my + 4) * (c->dc.mz + 4);
  delta2_kernel<<<grid_for(c, all), 256, 0, c->stream>>>(c->dc, c->aj, c->delta2);
  CB_CUDA(c, cudaGetLastError());
  if (c->cfg.precision == CB_MIXED)
    CB_CUDA(c, launch_mixed_prep(c->dc, (const double *const *)(c->ptab + PT_MET), c->delta2, c->aj, c->ptab4,
                                 c->ptab + PT_GCL, grid_for(c, (long long)c->plane), c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  c->have_grid = true;
  invalidate_graphs(c);
  return CB_OK;
}

int cb_get_metrics(cb_ctx *c, double *csi, double *eta, double *zet, double *aj) {
  if (!c || !csi || !eta || !zet || !aj) return CB_E_ARG;
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  double *outs[4] = {csi, eta, zet, aj};
  const int firsts[4] = {PT_MET + 0, PT_MET + 3, PT_MET + 6, PT_MISC + 0};
  const int ncs[4] = {3, 3, 3, 1};
  for (int f = 0; f < 4; f++) {
    pack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + firsts[f]),
                                                                     ncs[f], c->staging);
    CB_CUDA(c, cudaGetLastError());
    CB_CUDA(c, cudaMemcpyAsync(outs[f], c->staging, sizeof(double) * ncs[f] * nn, cudaMemcpyDeviceToHost, c->stream));
    CB_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return CB_OK;
}

int cb_set_nvert(cb_ctx *c, const double *nvert) {
  if (!c || !nvert) return CB_E_ARG;
  int e = upload_planes(c, nvert, 1, PT_MISC + 1, false);
  if (e) return e;
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  const int q = nvert_codes_exact(nvert, nn);
  bool zero = true;
  for (size_t t = 0; t < nn && zero; t++) zero = nvert[t] == 0.0;
  const bool nv0 = zero && !c->cfg.visT;  // the no-IBM variants carry no Sutherland law
  if (q != c->dc.nvq || nv0 != c->nv0 || zero != c->nvz) {
    c->dc.nvq = q;
    c->nv0 = nv0;
    c->nvz = zero;
    invalidate_graphs(c);  // the graphs carry the config and the kernel variant
  }
  return CB_OK;
}

// Mixed form: the reference state subtracted before FP32 rounding, the means
// of p, rhoE and T=p/rho over the owned nodes of the first uploaded state.
static void set_reference_state(cb_ctx *c, const double *q) {
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  double sp = 0, se = 0, st = 0;
  for (size_t t = 0; t < nn; t++) {
    const double *v = q + 5 * t;
    const double p = (c->cfg.gamma - 1) * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0]);
    sp += p;
    se += v[4];
    st += p / v[0];
  }
  c->dc.p_ref = sp / nn;
  c->dc.e_ref = se / nn;
  c->dc.t_ref = st / nn;
  c->dc.h_ref = c->dc.e_ref + c->dc.p_ref;
  c->have_refs = true;
  invalidate_graphs(c);
}

int cb_upload_state(cb_ctx *c, const double *q) {
  if (!c || !q) return CB_E_ARG;
  if (c->cfg.precision == CB_MIXED && !c->have_refs) set_reference_state(c, q);
  c->cur = 0;
  c->uc = -1;
  c->p_carry = false;
  int e = upload_planes(c, q, 5, PT_Q0, false);
  if (e) return e;
  CB_CUDA(c, cudaMemsetAsync(c->nut, 0, sizeof(double) * c->plane, c->stream));
  c->have_state = true;
  return CB_OK;
}

// Copy streams, staging buffers and events of the asynchronous transfers
// (once per context).
static int xfer_init(cb_ctx *c) {
  if (c->up_stream) return CB_OK;
  const size_t bytes = sizeof(double) * 5 * (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  CB_CUDA(c, cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking));
  CB_CUDA(c, cudaStreamCreateWithFlags(&c->down_stream, cudaStreamNonBlocking));
  for (int i = 0; i < 2; i++) {
    CB_CUDA(c, cudaMalloc(&c->stg_in[i], bytes));
    CB_CUDA(c, cudaMalloc(&c->stg_out[i], bytes));
    for (cudaEvent_t *e : {&c->ev_in_copied[i], &c->ev_in_free[i], &c->ev_out_ready[i], &c->ev_out_done[i]})
      CB_CUDA(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  return CB_OK;
}

int cb_upload_state_async(cb_ctx *c, const double *q) {
  if (!c || !q) return CB_E_ARG;
  int e = xfer_init(c);
  if (e) return e;
  if (c->cfg.precision == CB_MIXED && !c->have_refs) set_reference_state(c, q);
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  const int i = c->in_slot;
  c->in_slot ^= 1;
  // the copy into staging buffer i waits until its previous contents were unpacked
  CB_CUDA(c, cudaStreamWaitEvent(c->up_stream, c->ev_in_free[i], 0));
  CB_CUDA(c, cudaMemcpyAsync(c->stg_in[i], q, sizeof(double) * 5 * nn, cudaMemcpyHostToDevice, c->up_stream));
  CB_CUDA(c, cudaEventRecord(c->ev_in_copied[i], c->up_stream));
  // the state update itself is ordered on the compute stream, as cb_upload_state's
  CB_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_in_copied[i], 0));
  c->cur = 0;
  c->uc = -1;
  c->p_carry = false;
  unpack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, c->stg_in[i], 5, c->ptab + PT_Q0);
  CB_CUDA(c, cudaGetLastError());
  const long long all = (long long)(c->dc.mx + 4) * (c->dc.my + 4) * (c->dc.mz + 4);
  ghost_fill_kernel<<<grid_for(c, all), 256, 0, c->stream>>>(c->dc, c->ptab + PT_Q0, 5);
  CB_CUDA(c, cudaGetLastError());
  CB_CUDA(c, cudaEventRecord(c->ev_in_free[i], c->stream));
  CB_CUDA(c, cudaMemsetAsync(c->nut, 0, sizeof(double) * c->plane, c->stream));
  c->have_state = true;
  return CB_OK;
}

int cb_download_state_async(cb_ctx *c, double *q) {
  if (!c || !q) return CB_E_ARG;
  if (!c->have_state) return fail(c, CB_E_STATE, "no state uploaded");
  int e = xfer_init(c);
  if (e) return e;
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  const int o = c->out_slot;
  c->out_slot ^= 1;
  // the pack into staging buffer o waits until its previous copy to the host finished
  CB_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_out_done[o], 0));
  pack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + 5 * c->cur), 5,
                                                                   c->stg_out[o]);
  CB_CUDA(c, cudaGetLastError());
  CB_CUDA(c, cudaEventRecord(c->ev_out_ready[o], c->stream));
  CB_CUDA(c, cudaStreamWaitEvent(c->down_stream, c->ev_out_ready[o], 0));
  CB_CUDA(c, cudaMemcpyAsync(q, c->stg_out[o], sizeof(double) * 5 * nn, cudaMemcpyDeviceToHost, c->down_stream));
  CB_CUDA(c, cudaEventRecord(c->ev_out_done[o], c->down_stream));
  return CB_OK;
}

int cb_join_transfers(cb_ctx *c) {
  if (!c) return CB_E_ARG;
  if (!c->up_stream) return CB_OK;
  for (int i = 0; i < 2; i++) CB_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_out_done[i], 0));
  return CB_OK;
}

int cb_download_state(cb_ctx *c, double *q, double *p) {
  if (!c || !q) return CB_E_ARG;
  if (!c->have_state) return fail(c, CB_E_STATE, "no state uploaded");
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  pack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + 5 * c->cur), 5, c->staging);
  CB_CUDA(c, cudaGetLastError());
  CB_CUDA(c, cudaMemcpyAsync(q, c->staging, sizeof(double) * 5 * nn, cudaMemcpyDeviceToHost, c->stream));
  if (p) {
    CB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->p_carry)  // P as the interpolation and FormBCS(user, 0) left it
      pack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + PT_PL), 1,
                                                                      c->staging);
    else
      eos_pack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + 5 * c->cur), c->staging);
    CB_CUDA(c, cudaGetLastError());
    CB_CUDA(c, cudaMemcpyAsync(p, c->staging, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
  }
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

int cb_rhs(cb_ctx *c, int istage, double *rhs) {
  if (!c || !rhs) return CB_E_ARG;
  if (!c->have_state || !c->have_grid) return fail(c, CB_E_STATE, "grid and state must be set before cb_rhs");
  if (!c->rhsb[0]) {
    double *b = nullptr;
    CB_CUDA(c, cudaMalloc(&b, sizeof(double) * c->plane * 5));
    CB_CUDA(c, cudaMemsetAsync(b, 0, sizeof(double) * c->plane * 5, c->stream));
    for (int q = 0; q < 5; q++) c->rhsb[q] = b + c->plane * q;
    int e = fill_ptab(c);
    if (e) return e;
  }
  double alfa, beta;
  rk_coeffs(c, istage < 0 ? 0 : (istage > 2 ? 2 : istage), &alfa, &beta);
  DevFields F = fields_for(c, c->cur, c->cur, -1);
  if (c->p_carry) F.pin = c->pl;
  if (istage == 0) {
    int e = sigma_update(c, c->cur, c->p_carry ? c->pl : nullptr);
    if (e) return e;
  }
  CB_CUDA(c, launch_stage(c, F, istage, alfa, beta, 0.0, true));
  if (!c->cfg.inviscid) c->uc = c->cur;
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  pack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + PT_RHS), 5, c->staging);
  CB_CUDA(c, cudaGetLastError());
  CB_CUDA(c, cudaMemcpyAsync(rhs, c->staging, sizeof(double) * 5 * nn, cudaMemcpyDeviceToHost, c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

int cb_cfl_dt(cb_ctx *c, double cfl, double *dt, double *lambda_max) {
  if (!c || !dt || !(cfl > 0)) return CB_E_ARG;
  if (!c->have_state || !c->have_grid) return fail(c, CB_E_STATE, "grid and state must be set");
  unsigned long long *d = reinterpret_cast<unsigned long long *>(c->staging);  // staging is free between calls
  CB_CUDA(c, cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->stream));
  const long long work = (long long)(c->dc.mx - 2) * (c->dc.my - 2) * (c->dc.mz - 2);
  spectral_radius_kernel<<<grid_for(c, work), 256, 0, c->stream>>>(
      c->dc, (const double *const *)(c->ptab + 5 * c->cur), (const double *const *)(c->ptab + PT_MET), c->aj, c->nvert, d);
  CB_CUDA(c, cudaGetLastError());
  unsigned long long bits = 0;
  CB_CUDA(c, cudaMemcpyAsync(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  double lam;
  std::memcpy(&lam, &bits, sizeof(lam));
  if (lambda_max) *lambda_max = lam;
  *dt = lam > 0 ? cfl / lam : 0.0;
  return CB_OK;
}

int cb_calc_ucat(cb_ctx *c) {
  if (!c) return CB_E_ARG;
  if (!c->have_state) return fail(c, CB_E_STATE, "no state");
  c->uc = c->cur;
  return CB_OK;
}

int cb_eddy_viscosity(cb_ctx *c) {
  if (!c) return CB_E_ARG;
  if (!c->have_state || !c->have_grid) return fail(c, CB_E_STATE, "grid and state must be set");
  if (!c->cfg.les) return fail(c, CB_E_ARG, "eddy viscosity needs les != 0");
  int e = nut_update(c);
  if (e) return e;
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

int cb_get_nut(cb_ctx *c, double *nut) {
  if (!c || !nut) return CB_E_ARG;
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  pack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + PT_NUT), 1, c->staging);
  CB_CUDA(c, cudaGetLastError());
  CB_CUDA(c, cudaMemcpyAsync(nut, c->staging, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

int cb_get_cs(cb_ctx *c, double *cs) {
  if (!c || !cs) return CB_E_ARG;
  if (!c->dyn_arena) return fail(c, CB_E_STATE, "the coefficient plane exists with a dynamic les (>= 2, not 10) only");
  const size_t nn = (size_t)c->cfg.mx * c->cfg.my * c->cfg.mz;
  pack_kernel<<<grid_for(c, (long long)nn), 256, 0, c->stream>>>(c->dc, (const double *const *)(c->ptab + PT_DYN + 12), 1,
                                                                  c->staging);
  CB_CUDA(c, cudaGetLastError());
  CB_CUDA(c, cudaMemcpyAsync(cs, c->staging, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

int cb_rk_step(cb_ctx *c, int nsteps) {
  if (!c || nsteps < 0) return CB_E_ARG;
  if (!c->have_state || !c->have_grid) return fail(c, CB_E_STATE, "grid and state must be set before cb_rk_step");
  for (int n = 0; n < nsteps; n++) {
    const int ucslot = c->uc + 1;  // 0: none, 1..3: buffer
    GraphSlot &g = c->graphs[c->cur][ucslot][c->p_carry ? 1 : 0];
    if (c->use_graphs && !c->timing && g.exec) {
      const int ns = c->cfg.fluxorder;
      CB_CUDA(c, cudaGraphLaunch(g.exec, c->stream));
      // replay the bookkeeping of enqueue_step
      const int A = (c->cur + 1) % 3, B = (c->cur + 2) % 3;
      int in = c->cur;
      for (int s = 0; s < ns; s++) {
        const int out = (s % 2 == 0) ? A : B;
        if (!c->cfg.inviscid) c->uc = in;
        in = out;
      }
      c->cur = in;
      c->p_carry = ibm_active(c);
      continue;
    }
    if (c->use_graphs && !c->timing) {
      // capture this rotation state once, then replay it
      const int cur0 = c->cur, uc0 = c->uc;
      cudaGraph_t graph;
      CB_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int e = enqueue_step(c);
      cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
      if (e) return e;
      if (ce != cudaSuccess) return fail(c, CB_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return fail(c, CB_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
      (void)cur0; (void)uc0;
      CB_CUDA(c, cudaGraphLaunch(g.exec, c->stream));
      continue;
    }
    int e = enqueue_step(c);
    if (e) return e;
  }
  return CB_OK;
}

// Autotuner of the stage kernel's k-chunk (planes per block along k): times
// one stage launch per candidate on the current state, writing a buffer that
// holds neither the state nor the recorded velocity field, and keeps the
// fastest.  ncand = 0: every k-chunk from 4 to mz-2 that changes the number
// of chunks.  ms_out (optional, ncand entries or the default count) receives
// the average time of each candidate; *best the chosen k-chunk.
int cb_autotune(cb_ctx *c, int ncand, const int *cand, double *ms_out, int *nout, int *best) {
  if (!c || ncand < 0 || (ncand && !cand)) return CB_E_ARG;
  if (!c->have_state || !c->have_grid) return fail(c, CB_E_STATE, "grid and state must be set");
  std::vector<int> cs;
  const int nk = c->dc.mz - 2;
  if (ncand) {
    for (int t = 0; t < ncand; t++)
      if (cand[t] < 0) return fail(c, CB_E_ARG, "k-chunk candidates must be >= 0 (0: balanced segments)");
    cs.assign(cand, cand + ncand);
  } else {
    int last = -1;
    for (int kc = nk; kc >= 4; kc--) {
      const int ch = (nk + kc - 1) / kc;
      if (ch != last) { cs.push_back(kc); last = ch; }
    }
    cs.push_back(0);  // balanced segments, one range per resident CTA
  }
  const int in = c->cur;
  int out = (c->cur + 1) % 3;
  if (out == c->uc) out = (c->cur + 2) % 3;
  DevFields F = fields_for(c, in, in, out);
  cudaEvent_t e0, e1;
  CB_CUDA(c, cudaEventCreate(&e0));
  CB_CUDA(c, cudaEventCreate(&e1));
  const int keep = c->kchunk;
  double bms = 1e30, seg_ms = 1e30;
  int bkc = keep;
  for (size_t t = 0; t < cs.size(); t++) {
    c->kchunk = cs[t];
    float tot = 0.f;
    for (int rep = 0; rep < 3; rep++) {
      cudaEventRecord(e0, c->stream);
      cudaError_t ce = launch_stage(c, F, 1, 1.0, 1.0, 0.0, false);
      cudaEventRecord(e1, c->stream);
      if (ce != cudaSuccess) { c->kchunk = keep; return fail(c, CB_E_CUDA, cudaGetErrorString(ce)); }
      CB_CUDA(c, cudaEventSynchronize(e1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep) tot += ms;  // the first launch warms the caches
    }
    const double avg = tot / 2.0;
    if (ms_out && (!nout || (int)t < *nout)) ms_out[t] = avg;
    if (cs[t] == 0) seg_ms = avg;
    else if (avg < bms) { bms = avg; bkc = cs[t]; }
  }
  // the balanced segments read more DRAM (their halo planes are less often
  // shared through L2 at 130^3: 1.4x more bytes per launch); they are kept
  // only when clearly faster than the best chunked grid
  if (seg_ms < 0.97 * bms) { bms = seg_ms; bkc = 0; }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (nout) *nout = (int)cs.size();
  c->kchunk = bkc;
  if (best) *best = bkc;
  invalidate_graphs(c);  // the graphs carry the launch shape
  return CB_OK;
}

int cb_capture_graph(cb_ctx *c) {
  if (!c) return CB_E_ARG;
  if (!c->have_state || !c->have_grid) return fail(c, CB_E_STATE, "grid and state must be set");
  c->use_graphs = true;
  return CB_OK;
}

// ------------------------------------------------------ immersed boundary --
static int ibm_body(cb_ctx *c, int ibi, IbmBody **b) {
  if (!c) return CB_E_ARG;
  if (ibi < 0 || ibi >= CB_IBM_MAX_BODIES) return fail(c, CB_E_ARG, "body index out of range");
  *b = &c->ibm[ibi];
  return CB_OK;
}

int cb_ibm_set_surface(cb_ctx *c, int ibi, int n_v, int n_elmt, const int *nv1, const int *nv2, const int *nv3,
                       const double *nf_x, const double *nf_y, const double *nf_z) {
  IbmBody *b;
  int e = ibm_body(c, ibi, &b);
  if (e) return e;
  if (n_v < 1 || n_elmt < 1 || !nv1 || !nv2 || !nv3 || !nf_x || !nf_y || !nf_z)
    return fail(c, CB_E_ARG, "surface needs n_v, n_elmt >= 1 and all arrays");
  CB_CUDA(c, cudaStreamSynchronize(c->stream));  // graphs in flight may read the old arrays
  ibm_drop_list(*b);
  if (b->surf) cudaFree(b->surf);
  b->surf = nullptr;
  const char *err = "";
  const int rc = ibm_surface_to_device(*b, n_v, n_elmt, nv1, nv2, nv3, nf_x, nf_y, nf_z, c->stream, &err);
  if (rc == CB_E_ARG) return fail(c, CB_E_ARG, err);
  if (rc) return fail(c, CB_E_CUDA, "surface upload");
  invalidate_graphs(c);
  return CB_OK;
}

int cb_ibm_set_velocity(cb_ctx *c, int ibi, const double *u, const double *uold) {
  IbmBody *b;
  int e = ibm_body(c, ibi, &b);
  if (e) return e;
  if (!u || !uold) return CB_E_ARG;
  if (!b->surf) return fail(c, CB_E_STATE, "set the body's surface first");
  // stream-ordered: steps enqueued before this call read the previous values
  CB_CUDA(c, cudaMemcpyAsync(b->u, u, sizeof(double) * 3 * b->n_v, cudaMemcpyHostToDevice, c->stream));
  CB_CUDA(c, cudaMemcpyAsync(b->uold, uold, sizeof(double) * 3 * b->n_v, cudaMemcpyHostToDevice, c->stream));
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

int cb_ibm_set_list(cb_ctx *c, int ibi, int n, const cb_ibm_info *list, const double *coor) {
  IbmBody *b;
  int e = ibm_body(c, ibi, &b);
  if (e) return e;
  if (n < 0 || (n > 0 && (!list || !coor))) return CB_E_ARG;
  if (n > 0 && !b->surf) return fail(c, CB_E_STATE, "set the body's surface first");
  IbmHostList h;
  const char *err = "";
  if (ibm_build_list(c->dc, c->cfg.isothermal == 2, b->n_elmt, n, list, coor, h, &err)) return fail(c, CB_E_ARG, err);
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  ibm_drop_list(*b);
  invalidate_graphs(c);
  if (h.n() == 0) return CB_OK;
  if (!c->ibm_arena) {
    CB_CUDA(c, cudaMalloc(&c->ibm_arena, sizeof(double) * 7 * c->plane));
    CB_CUDA(c, cudaMemsetAsync(c->ibm_arena, 0, sizeof(double) * 7 * c->plane, c->stream));
    c->spare = c->ibm_arena;
    c->psnap = c->ibm_arena + 5 * c->plane;
    c->pl = c->ibm_arena + 6 * c->plane;
    int fe = fill_ptab(c);
    if (fe) return fe;
  }
  const cudaError_t le = ibm_list_to_device(*b, h, c->stream);
  if (le != cudaSuccess) {  // no half-uploaded list stays behind
    ibm_drop_list(*b);
    return fail(c, CB_E_CUDA, std::string("list upload: ") + cudaGetErrorString(le));
  }
  return CB_OK;
}

int cb_ibm_count(const cb_ctx *c, int ibi) {
  if (!c || ibi < 0 || ibi >= CB_IBM_MAX_BODIES) return -1;
  return c->ibm[ibi].n;
}

int cb_ibm_set_options(cb_ctx *c, int twoD, int wallfunction) {
  if (!c) return CB_E_ARG;
  if (twoD < 0 || twoD > 3) return fail(c, CB_E_ARG, "twoD must be 0..3");
  // wallfunction 1 reads a table that pre_integrate builds in a stack array of
  // its own frame (wallfunction.c:113-145): its values are undefined
  if (wallfunction == 1) return fail(c, CB_E_UNSUPPORTED, "the wall function of -wallfunction 1 is not built");
  if (wallfunction != 0 && wallfunction != 2 && wallfunction != 3)
    return fail(c, CB_E_ARG, "wallfunction must be 0, 2 or 3");
  c->ibm_twoD = twoD;
  c->ibm_wallfunction = wallfunction;
  invalidate_graphs(c);
  return CB_OK;
}

int cb_ibm_get_ustar(cb_ctx *c, int ibi, double *ustar) {
  IbmBody *b;
  int e = ibm_body(c, ibi, &b);
  if (e) return e;
  if (b->n > 0) {
    if (!ustar) return fail(c, CB_E_ARG, "null ustar");
    CB_CUDA(c, cudaMemcpyAsync(ustar, b->ustar, sizeof(double) * b->n, cudaMemcpyDeviceToHost, c->stream));
    CB_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return CB_OK;
}

int cb_ibm_interpolate(cb_ctx *c, int ibi, int add_dundt) {
  IbmBody *b;
  int e = ibm_body(c, ibi, &b);
  if (e) return e;
  if (!c->have_state) return fail(c, CB_E_STATE, "no state uploaded");
  if (b->n > 0) {
    if (!c->p_carry) {  // P is the EqOfState of the state until an interpolation writes it
      e = eos_to_plane(c);
      if (e) return e;
    }
    // Qold between steps is the state itself (main.c:971 copies Q to Qold
    // after every step); the sweeps rewrite the state, so -isothermal 2 reads
    // a copy of its density taken first
    const double *rho_old = nullptr;
    if (c->cfg.isothermal == 2) {
      CB_CUDA(c, cudaMemcpyAsync(c->spare, c->qb[c->cur][0], sizeof(double) * c->plane, cudaMemcpyDeviceToDevice,
                                 c->stream));
      rho_old = c->spare;
    }
    e = ibm_sweeps(c, *b, add_dundt ? 1 : 0, rho_old);
    if (e) return e;
    c->p_carry = true;
  }
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  return CB_OK;
}

int cb_sync(cb_ctx *c) {
  if (!c) return CB_E_ARG;
  CB_CUDA(c, cudaStreamSynchronize(c->stream));
  unsigned st = 0;
  CB_CUDA(c, cudaMemcpy(&st, c->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (st) {
    CB_CUDA(c, cudaMemset(c->status, 0, sizeof(unsigned)));
    char buf[160];
    snprintf(buf, sizeof(buf), "device status 0x%x:%s%s%s", st, (st & ST_NONFINITE) ? " non-finite" : "",
             (st & ST_NEG_RHO) ? " rho<=0" : "", (st & ST_NEG_P) ? " p<=0" : "");
    return fail(c, CB_E_NONFINITE, buf);
  }
  return CB_OK;
}

int cb_timing_enable(cb_ctx *c, int on) {
  if (!c) return CB_E_ARG;
  harvest_timing(c);
  c->timing = on != 0;
  c->acc_rhs_ms = c->acc_other_ms = 0;
  c->acc_rhs_n = c->acc_other_n = 0;
  return CB_OK;
}

int cb_timing_read(cb_ctx *c, double *rhs_ms, int *rhs_n, double *other_ms, int *other_n) {
  if (!c) return CB_E_ARG;
  harvest_timing(c);
  if (rhs_ms) *rhs_ms = c->acc_rhs_ms;
  if (rhs_n) *rhs_n = c->acc_rhs_n;
  if (other_ms) *other_ms = c->acc_other_ms;
  if (other_n) *other_n = c->acc_other_n;
  return CB_OK;
}

}  // extern "C"
