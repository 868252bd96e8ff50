// Batched multi-block form: many curvilinear blocks of uneven sizes resident
// on one GPU and advanced together.
//
// Layout: every field is ONE contiguous array over all blocks' padded node
// boxes (block b at offset off[b]), so a node is addressed by a single global
// offset valid in every field and every state buffer.  That lets one gather
// table describe all inter-block halo copies:
//   entry = (dst offset, src offset, source buffer)
// where the source buffer is the stage output (a donor's freshly updated
// interior) or the stage input (the reference's periodic FormBCS, which reads
// the not-yet-refreshed lQ, rhs.c:1107-1227).
//
// Per RK stage: ONE persistent stage launch over a largest-first list of work
// items (block, tile column, k-chunk) taken from a device counter, then one
// gather launch.  The eddy viscosity runs once per step per block.  A whole
// step is captured as a CUDA graph per buffer-rotation state.  The k-chunk of
// the work items is chosen by timing candidates (cb_batch_autotune).  For
// comparison the same step can run with one stage launch per block.
//
// The reference advances its blocks one after another without coupling
// (solvers.c:246); the gather is new.  With the self-periodic map
// (cb_batch_halo_periodic) every block reproduces the single-block path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
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

// gather: dst[e] <- (from_in[e] ? qin : qout)[src[e]] for the 5 state fields
__global__ void halo_gather_kernel(const long long *__restrict__ dst, const long long *__restrict__ src,
                                   const unsigned char *__restrict__ from_in, long long n, DevFields F) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long d = dst[e], s = src[e];
    const bool fin = from_in[e] != 0;
#pragma unroll
    for (int q = 0; q < 5; q++) F.qout[q][d] = fin ? F.q[q][s] : F.qout[q][s];
  }
}

// single-field gather within one array: dst[e] <- f[src[e]] (plain periodic
// wrap / DMGlobalToLocal across blocks: the eddy viscosity and the initial state)
__global__ void plane_gather_kernel(const long long *__restrict__ dst, const long long *__restrict__ src, long long n,
                                    double *f) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    f[dst[e]] = f[src[e]];
}

// Cross-process halo exchange: pack the values this process owes its peers
// into a caller-owned device buffer (entry-major, nf values per entry) and
// scatter the values received from them.
struct FieldSet {
  const double *in[5];
  const double *out[5];
};
struct OutSet {
  double *a[5];
};
__global__ void xpack_kernel(const long long *__restrict__ src, const unsigned char *__restrict__ fin, long long n, int nf,
                             FieldSet fs, double *__restrict__ buf) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long sidx = src[e];
    const bool from_in = fin != nullptr && fin[e] != 0;
    for (int f = 0; f < nf; f++) buf[e * nf + f] = from_in ? fs.in[f][sidx] : fs.out[f][sidx];
  }
}
__global__ void xunpack_kernel(const long long *__restrict__ dst, long long n, int nf, OutSet os,
                               const double *__restrict__ buf) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long d = dst[e];
    for (int f = 0; f < nf; f++) os.a[f][d] = buf[e * nf + f];
  }
}

struct Xchg {
  long long nsend = 0, nrecv = 0;
  long long *d_src = nullptr, *d_dst = nullptr;
  unsigned char *d_fin = nullptr;
  double *d_send = nullptr, *d_recv = nullptr;  // caller-owned
};

struct BlockHost {
  int mx, my, mz;
  DevCfg dc;
  long long off;        // offset of the block's padded box in every field array
  int tiles_x, tiles_y;
  bool have_grid = false, have_state = false;
  bool nvz = true;      // the block's nvert is zero everywhere
  bool phys = false;    // a physical face code: the block runs its own FormBCS
};

}  // namespace

struct cb_batch {
  cb_config cfg{};
  int nb = 0;
  int dev = 0, sms = 148;
  cudaStream_t stream = nullptr;
  std::vector<BlockHost> blk;
  long long total = 0;  // padded nodes over all blocks
  // fields (each `total` long): 3 x 5 state, 9 metrics, aj, nvert, nut, delta2
  double *arena = nullptr;
  double *qb[3][5] = {};
  double *met[3][3] = {};
  double *aj = nullptr, *nvert = nullptr, *nut = nullptr, *delta2 = nullptr;
  // shock sensor (calc_sigma): the hybrid weights (s_x, s_y, s_z) and the
  // planes of the filter pass, each `total` long; per block a device table of
  // its six plane pointers (weights, then filter planes)
  double *sig_arena = nullptr;
  double *sig_a[3] = {}, *sig_b[3] = {};
  double **d_sigptr = nullptr;
  // immersed bodies (blocks with face codes only): the bodies' surfaces; per
  // block its list of each body, its seven planes (Q snapshot 5, P snapshot,
  // the carried P) and a device table of their pointers
  IbmBody body[CB_IBM_MAX_BODIES];
  std::vector<IbmBody> ibl;        // [nb][CB_IBM_MAX_BODIES]: list part (the surface is body[ibi]'s)
  std::vector<double *> ib_arena;  // per block: 7 planes of its padded box, or null
  double **d_ibtab = nullptr;      // [nb][7]
  int ibm_twoD = 0, ibm_wallfunction = 0;
  // k-lo inflow codes 52 and 47: per block its node coordinates x, y (two
  // padded planes, or null), and the step index user->ti of the running step
  std::vector<double *> coorxy;
  int *ti_dev = nullptr;
  // dynamic Smagorinsky model (-les 2/3): 14 planes, each `total` long, and
  // per block a device table of its 14 plane pointers
  double *dyn_arena = nullptr;
  double **d_dynptr = nullptr;
  double dyn_tf_mult = 2.0;
  void *arena_mixed = nullptr;
  float4 *met4[3] = {};
  double *gcl[3] = {};
  double *staging = nullptr;  // AoS host transfer buffer, sized for the largest block
  double **ptab = nullptr;    // per-block pointer tables for the set-up kernels
  float4 **ptab4 = nullptr;
  // batched launch data
  BatchBlock *d_tables = nullptr;  // [27][nb] indexed by (in, old, out) buffer triple
  int2 *d_items = nullptr;
  int nitems = 0;
  unsigned *d_counter = nullptr;
  unsigned *status = nullptr;
  int kchunk = 16;
  // stage halo map (FormBCS + wrap across blocks) and plain wrap map
  long long nhalo = 0, nwrap = 0;
  long long *d_hdst = nullptr, *d_hsrc = nullptr, *d_wdst = nullptr, *d_wsrc = nullptr;
  unsigned char *d_hin = nullptr;
  bool ghosts_dirty = false;  // uploaded state still carries per-block ghosts
  // blocks with a physical face code (cb_batch_set_bctype), and per map kind
  // the blocks that hold a destination of that map
  int nphys = 0;
  std::vector<char> map_dst[2];
  // cross-process exchange (stage values, wrap values) and the phase state
  Xchg xs, xw;
  int xcur0 = -1, xnext = 0, xin = -1, xout = -1;
  // stepping
  int cur = 0, uc = -1;
  cudaGraphExec_t graphs[2][3][4] = {};
  bool have_refs = false;
  std::string err;
};

// FLUX bits of the batch's stage kernels: Roe, WENO5-JS, and with LES the
// constant blend weight s_x = s_y = s_z when it is exactly 1 or 0 and the
// sensor is off (the single-block context's rule)
static int batch_flux_bits(const cb_config &f) {
  int fl = (f.flux == 1 ? FLUX_ROE : 0) | (f.weno_order == 5 ? FLUX_W5 : 0);
  if (f.les && !f.calc_sigma && f.s_x == f.s_y && f.s_y == f.s_z) {
    if (f.s_x == 1.0) fl |= FLUX_SIGMA1;
    else if (f.s_x == 0.0) fl |= FLUX_SIGMA0;
  }
  // block faces are interfaces (bctype 7): with no 2-D mode and MUSCL (or
  // WENO5-JS, whose reconstruction the W5 bit selects) the PLAIN variants
  if (f.twod == 0 && (f.fluxorder == 2 || f.weno_order == 5)) fl |= FLUX_PLAIN;
  return fl;
}

// -les 2, 3, ... (not 10): the dynamic model (Compute_Smagorinsky_Constant_1)
static bool batch_dynamic(const cb_config &f) { return f.les >= 2 && f.les != 10; }

// The bits the batch launches with: a block with a physical face code needs
// the boundary-code branches the PLAIN variants fold away.
static int batch_bits(const cb_batch *b) {
  const int fl = batch_flux_bits(b->cfg);
  return b->nphys ? (fl & ~FLUX_PLAIN) : fl;
}

// every block's nvert is zero: the stage kernels' no-IBM variant
static bool batch_nv0(const cb_batch *b) {
  if (b->cfg.visT) return false;  // the no-IBM variants carry no Sutherland law
  for (const auto &bh : b->blk)
    if (!bh.nvz) return false;
  return true;
}

static int bfail(cb_batch *b, int code, const std::string &m) {
  if (b) b->err = m;
  return code;
}
#define BCUDA(b, call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return bfail(b, CB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

static int bgrid(const cb_batch *b, long long work) {
  long long g = (work + 255) / 256, cap = (long long)b->sms * 8;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

static void destroy_graphs(cb_batch *b) {
  if (b->stream) cudaStreamSynchronize(b->stream);  // no graph is destroyed while it runs
  for (auto &m : b->graphs)
    for (auto &r : m)
      for (auto &g : r)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

// Block k holds an interpolation list of some body.
static bool block_ib(const cb_batch *b, int k) {
  if (b->ib_arena.empty() || !b->ib_arena[k]) return false;
  for (int i = 0; i < CB_IBM_MAX_BODIES; i++)
    if (b->ibl[(size_t)k * CB_IBM_MAX_BODIES + i].n > 0) return true;
  return false;
}
// the pressure plane block k carries from its interpolation into the next
// step's first stage (the reference's lP)
static double *ib_pl(const cb_batch *b, int k) { return b->ib_arena[k] + 6 * b->blk[k].dc.plane; }

// Pointers of one block (all fields at the block's offset) for a buffer
// triple; a first stage (in == old) of a block with bodies reads the carried
// pressure, as the single-block context does after an immersed step.
static DevFields block_fields(const cb_batch *b, int blk, int in, int old, int out) {
  const long long o = b->blk[blk].off;
  DevFields F{};
  for (int q = 0; q < 5; q++) {
    F.q[q] = b->qb[in][q] + o;
    F.qold[q] = b->qb[old][q] + o;
    F.qout[q] = out >= 0 ? b->qb[out][q] + o : nullptr;
    F.rhs[q] = nullptr;
  }
  for (int e = 0; e < 3; e++) {
    for (int q = 0; q < 3; q++) F.met[e][q] = b->met[e][q] + o;
    F.met4[e] = b->met4[e] ? b->met4[e] + o : nullptr;
  }
  F.aj = b->aj + o;
  F.nvert = b->nvert + o;
  F.nut = b->nut + o;
  F.delta2 = b->delta2 + o;
  for (int a = 0; a < 3; a++) F.gcl[a] = b->gcl[a] ? b->gcl[a] + o : nullptr;
  for (int a = 0; a < 3; a++) F.sig[a] = b->sig_a[a] ? b->sig_a[a] + o : nullptr;
  F.status = b->status;
  if (in == old && block_ib(b, blk)) F.pin = ib_pl(b, blk);
  const double *xy = b->coorxy.empty() ? nullptr : b->coorxy[blk];
  F.cx = xy;
  F.cy = xy ? xy + b->blk[blk].dc.plane : nullptr;
  F.ti = b->ti_dev;
  return F;
}

// Builds the 27 (in, old, out) tables and the largest-first item list.
static int build_tables(cb_batch *b) {
  std::vector<BatchBlock> h((size_t)27 * b->nb);
  for (int in = 0; in < 3; in++)
    for (int old = 0; old < 3; old++)
      for (int out = 0; out < 3; out++)
        for (int k = 0; k < b->nb; k++) {
          BatchBlock &t = h[(size_t)(in * 9 + old * 3 + out) * b->nb + k];
          const BlockHost &bh = b->blk[k];
          t.c = bh.dc;
          t.F = block_fields(b, k, in, old, out);
          t.tiles_x = bh.tiles_x;
          t.tiles_y = bh.tiles_y;
          t.kchunk = b->kchunk;
          t.nchunks = (bh.mz - 2 + b->kchunk - 1) / b->kchunk;
          t.first_item = 0;
        }
  // items: (block, local index), ordered by descending estimated cost
  struct It { int blk, loc; long long cost; };
  std::vector<It> items;
  for (int k = 0; k < b->nb; k++) {
    const BlockHost &bh = b->blk[k];
    const int nch = (bh.mz - 2 + b->kchunk - 1) / b->kchunk;
    for (int z = 0; z < nch; z++)
      for (int y = 0; y < bh.tiles_y; y++)
        for (int x = 0; x < bh.tiles_x; x++) {
          const int by = stage_tile_rows(batch_bits(b));
          const int nxn = std::min(SBX, bh.mx - 2 - x * SBX), nyn = std::min(by, bh.my - 2 - y * by);
          const int nzn = std::min(b->kchunk, bh.mz - 2 - z * b->kchunk);
          // interior nodes plus the 3-plane prologue of each chunk
          items.push_back({k, (z * bh.tiles_y + y) * bh.tiles_x + x, (long long)nxn * nyn * (nzn + 3)});
        }
  }
  std::stable_sort(items.begin(), items.end(), [](const It &a, const It &c) { return a.cost > c.cost; });
  std::vector<int2> hi(items.size());
  for (size_t i = 0; i < items.size(); i++) hi[i] = make_int2(items[i].blk, items[i].loc);
  if (b->d_items) cudaFree(b->d_items);
  b->d_items = nullptr;
  b->nitems = (int)hi.size();
  BCUDA(b, cudaMalloc(&b->d_items, sizeof(int2) * hi.size()));
  BCUDA(b, cudaMemcpy(b->d_items, hi.data(), sizeof(int2) * hi.size(), cudaMemcpyHostToDevice));
  if (!b->d_tables) BCUDA(b, cudaMalloc(&b->d_tables, sizeof(BatchBlock) * h.size()));
  BCUDA(b, cudaMemcpy(b->d_tables, h.data(), sizeof(BatchBlock) * h.size(), cudaMemcpyHostToDevice));
  destroy_graphs(b);
  return CB_OK;
}

static int block_ptab(cb_batch *b, int k) {
  // per-block pointer table for the set-up kernels (planes of block k)
  const long long o = b->blk[k].off;
  double *h[64] = {};
  for (int s = 0; s < 3; s++)
    for (int q = 0; q < 5; q++) h[5 * s + q] = b->qb[s][q] + o;
  for (int e = 0; e < 3; e++)
    for (int q = 0; q < 3; q++) h[15 + 3 * e + q] = b->met[e][q] + o;
  h[24] = b->aj + o;  // 15..24: 9 metrics + aj contiguous for the ghost fill
  h[25] = b->nvert + o;
  h[26] = b->nut + o;
  for (int a = 0; a < 3; a++) h[27 + a] = b->gcl[a] ? b->gcl[a] + o : nullptr;
  BCUDA(b, cudaMemcpyAsync(b->ptab, h, sizeof(h), cudaMemcpyHostToDevice, b->stream));
  if (b->ptab4) {
    float4 *h4[3] = {b->met4[0] + o, b->met4[1] + o, b->met4[2] + o};
    BCUDA(b, cudaMemcpyAsync(b->ptab4, h4, sizeof(h4), cudaMemcpyHostToDevice, b->stream));
  }
  BCUDA(b, cudaStreamSynchronize(b->stream));
  return CB_OK;
}

extern "C" {

int cb_batch_create(const cb_config *cfg, int nblocks, const int *dims, cb_batch **out) {
  if (!cfg || !dims || !out || nblocks < 1) return CB_E_ARG;
  *out = nullptr;
  cb_batch *b = new cb_batch();
  b->cfg = *cfg;
  b->nb = nblocks;
  auto bail = [&](int code, const char *m) {
    fprintf(stderr, "chimera_b200: cb_batch_create: %s\n", m);
    cb_batch_destroy(b);
    return code;
  };
  if (cfg->fluxorder < 1 || cfg->fluxorder > 3 || (cfg->eno_order != 2 && cfg->eno_order != 3) ||
      cfg->les < 0 || (cfg->precision != CB_FP64 && cfg->precision != CB_MIXED) ||
      (cfg->flux != 0 && cfg->flux != 1) ||
      (cfg->weno_order != 3 && cfg->weno_order != 5))
    return bail(CB_E_UNSUPPORTED, "option combination not built");
  if (cfg->weno_order == 5 && cfg->fluxorder != 3) return bail(CB_E_ARG, "weno_order 5 needs fluxorder 3");
  if (cfg->visT && !(cfg->tref > 0.0)) return bail(CB_E_ARG, "Tref must be > 0 with visT");
  if (batch_dynamic(*cfg) && !(cfg->max_cs >= 0.0)) return bail(CB_E_ARG, "max_cs must be >= 0");
  b->dev = cfg->device;
  if (cudaSetDevice(b->dev) != cudaSuccess) return bail(CB_E_CUDA, "cudaSetDevice");
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->dev);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(CB_E_CUDA, "stream");
  long long off = 0;
  size_t maxnn = 0;
  for (int k = 0; k < nblocks; k++) {
    BlockHost bh{};
    bh.mx = dims[3 * k]; bh.my = dims[3 * k + 1]; bh.mz = dims[3 * k + 2];
    if (bh.mx < 6 || bh.my < 6 || bh.mz < 6) return bail(CB_E_ARG, "every block needs at least 6 nodes per direction");
    DevCfg &d = bh.dc;
    d.mx = bh.mx; d.my = bh.my; d.mz = bh.mz;
    d.px = ((bh.mx + 4 + 15) / 16) * 16;
    d.py = bh.my + 4;
    d.pz = bh.mz + 4;
    d.plane = (long long)d.px * d.py * d.pz;
    for (int s = 0; s < 6; s++) d.bctype[s] = 7;  // block faces are interfaces: full-order stencils into the halo
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
    d.nvq = 1;  // nvert starts zero
    d.calc_sigma = (cfg->les && cfg->calc_sigma) ? 1 : 0;
    d.s_x_min = cfg->s_x_min; d.s_y_min = cfg->s_y_min; d.s_z_min = cfg->s_z_min;
    d.ks = cfg->sigma_thrsh;
    d.abc = cfg->abc;
    d.flux = cfg->flux;
    d.twall = cfg->twall;
    if (shell_count(d) >= (1LL << 31)) return bail(CB_E_ARG, "block too large for 32-bit boundary indexing");
    bh.off = off;
    off += (d.plane + 31) / 32 * 32;  // 256-byte aligned block starts
    bh.tiles_x = (bh.mx - 2 + SBX - 1) / SBX;
    const int by = stage_tile_rows(batch_flux_bits(*cfg));  // the variant's tile height
    bh.tiles_y = (bh.my - 2 + by - 1) / by;
    maxnn = std::max(maxnn, (size_t)bh.mx * bh.my * bh.mz);
    b->blk.push_back(bh);
  }
  b->total = off;
  b->ibl.resize((size_t)nblocks * CB_IBM_MAX_BODIES);
  b->ib_arena.assign(nblocks, nullptr);
  b->coorxy.assign(nblocks, nullptr);
  if (cudaMalloc(&b->ti_dev, sizeof(int)) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc step index");
  cudaMemsetAsync(b->ti_dev, 0, sizeof(int), b->stream);
  const size_t bytes = sizeof(double) * (size_t)b->total * 28;
  if (cudaMalloc(&b->arena, bytes) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc arena");
  cudaMemsetAsync(b->arena, 0, bytes, b->stream);
  int p = 0;
  for (int s = 0; s < 3; s++)
    for (int q = 0; q < 5; q++) b->qb[s][q] = b->arena + (size_t)b->total * (p++);
  for (int e = 0; e < 3; e++)
    for (int q = 0; q < 3; q++) b->met[e][q] = b->arena + (size_t)b->total * (p++);
  b->aj = b->arena + (size_t)b->total * (p++);
  b->nvert = b->arena + (size_t)b->total * (p++);
  b->nut = b->arena + (size_t)b->total * (p++);
  b->delta2 = b->arena + (size_t)b->total * (p++);
  if (cfg->precision == CB_MIXED) {
    const size_t mb = sizeof(float4) * (size_t)b->total * 3 + sizeof(double) * (size_t)b->total * 3;
    if (cudaMalloc(&b->arena_mixed, mb) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc mixed");
    cudaMemsetAsync(b->arena_mixed, 0, mb, b->stream);
    float4 *f = (float4 *)b->arena_mixed;
    for (int e = 0; e < 3; e++) b->met4[e] = f + (size_t)b->total * e;
    double *g = (double *)(f + (size_t)b->total * 3);
    for (int a = 0; a < 3; a++) b->gcl[a] = g + (size_t)b->total * a;
    if (cudaMalloc(&b->ptab4, sizeof(float4 *) * 3) != cudaSuccess) return bail(CB_E_CUDA, "ptab4");
  }
  if (batch_dynamic(*cfg)) {
    b->dyn_tf_mult = cfg->testfilter_ik ? pow(5.0, 1. / 3.) : 2.0;  // the host's pow, as the reference's
    if (cudaFuncSetAttribute(dyn_lm_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DYN_LM_SMEM) !=
        cudaSuccess)
      return bail(CB_E_CUDA, "dynamic-model kernel attributes");
    const size_t db = sizeof(double) * (size_t)b->total * 14;
    if (cudaMalloc(&b->dyn_arena, db) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc dynamic-model planes");
    cudaMemsetAsync(b->dyn_arena, 0, db, b->stream);
    std::vector<double *> hp((size_t)14 * nblocks);
    for (int k = 0; k < nblocks; k++)
      for (int a = 0; a < 14; a++) hp[14 * k + a] = b->dyn_arena + (size_t)b->total * a + b->blk[k].off;
    if (cudaMalloc(&b->d_dynptr, sizeof(double *) * hp.size()) != cudaSuccess) return bail(CB_E_CUDA, "dynamic table");
    if (cudaMemcpy(b->d_dynptr, hp.data(), sizeof(double *) * hp.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(CB_E_CUDA, "dynamic table");
  }
  if (cfg->les && cfg->calc_sigma) {
    const size_t sb = sizeof(double) * (size_t)b->total * 6;
    if (cudaMalloc(&b->sig_arena, sb) != cudaSuccess) return bail(CB_E_CUDA, "cudaMalloc sensor planes");
    cudaMemsetAsync(b->sig_arena, 0, sb, b->stream);
    for (int a = 0; a < 3; a++) {
      b->sig_a[a] = b->sig_arena + (size_t)b->total * a;
      b->sig_b[a] = b->sig_arena + (size_t)b->total * (3 + a);
    }
    std::vector<double *> hp((size_t)6 * nblocks);
    for (int k = 0; k < nblocks; k++)
      for (int a = 0; a < 3; a++) {
        hp[6 * k + a] = b->sig_a[a] + b->blk[k].off;
        hp[6 * k + 3 + a] = b->sig_b[a] + b->blk[k].off;
      }
    if (cudaMalloc(&b->d_sigptr, sizeof(double *) * hp.size()) != cudaSuccess) return bail(CB_E_CUDA, "sensor table");
    if (cudaMemcpy(b->d_sigptr, hp.data(), sizeof(double *) * hp.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(CB_E_CUDA, "sensor table");
  }
  {
    const bool mix = cfg->precision == CB_MIXED;
    if (stage_attrs_all(mix) != cudaSuccess || batch_attrs_all(mix) != cudaSuccess)
      return bail(CB_E_CUDA, "stage kernel attributes");
  }
  if (cudaMalloc(&b->staging, sizeof(double) * 5 * maxnn) != cudaSuccess) return bail(CB_E_CUDA, "staging");
  if (cudaMalloc(&b->ptab, sizeof(double *) * 64) != cudaSuccess) return bail(CB_E_CUDA, "ptab");
  if (cudaMalloc(&b->d_counter, sizeof(unsigned)) != cudaSuccess) return bail(CB_E_CUDA, "counter");
  if (cudaMalloc(&b->status, sizeof(unsigned)) != cudaSuccess) return bail(CB_E_CUDA, "status");
  cudaMemsetAsync(b->status, 0, sizeof(unsigned), b->stream);
  if (build_tables(b)) return bail(CB_E_CUDA, b->err.c_str());
  *out = b;
  return CB_OK;
}

void cb_batch_destroy(cb_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  destroy_graphs(b);
  for (auto &l : b->ibl) ibm_drop_list(l);
  for (auto &s : b->body)
    if (s.surf) cudaFree(s.surf);
  for (double *p : b->ib_arena)
    if (p) cudaFree(p);
  for (double *p : b->coorxy)
    if (p) cudaFree(p);
  if (b->ti_dev) cudaFree(b->ti_dev);
  if (b->d_ibtab) cudaFree(b->d_ibtab);
  void *ptrs[] = {b->arena, b->arena_mixed, b->sig_arena, b->d_sigptr, b->dyn_arena, b->d_dynptr, b->staging, b->ptab,
                  b->ptab4, b->d_tables,
                  b->d_items, b->d_counter,
                  b->status, b->d_hdst, b->d_hsrc, b->d_hin, b->d_wdst, b->d_wsrc,
                  b->xs.d_src, b->xs.d_dst, b->xs.d_fin, b->xw.d_src, b->xw.d_dst, b->xw.d_fin};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

const char *cb_batch_last_error(const cb_batch *b) { return b ? b->err.c_str() : "null batch"; }
long long cb_batch_interior_nodes(const cb_batch *b) {
  long long s = 0;
  if (b)
    for (auto &bh : b->blk) s += (long long)(bh.mx - 2) * (bh.my - 2) * (bh.mz - 2);
  return s;
}
void *cb_batch_stream(cb_batch *b) { return b ? (void *)b->stream : nullptr; }
int cb_batch_work_items(const cb_batch *b) { return b ? b->nitems : 0; }

static int check_block(cb_batch *b, int k) {
  if (!b || k < 0 || k >= b->nb) return CB_E_ARG;
  return CB_OK;
}

int cb_batch_set_grid(cb_batch *b, int k, const double *coor) {
  if (check_block(b, k) || !coor) return CB_E_ARG;
  BlockHost &bh = b->blk[k];
  const DevCfg &d = bh.dc;
  const size_t nn = (size_t)bh.mx * bh.my * bh.mz;
  if (block_ptab(b, k)) return CB_E_CUDA;
  BCUDA(b, cudaMemcpyAsync(b->staging, coor, sizeof(double) * 3 * nn, cudaMemcpyHostToDevice, b->stream));
  // coordinates into the block's state buffer 2 (scratch until a state is uploaded)
  unpack_kernel<<<bgrid(b, (long long)nn), 256, 0, b->stream>>>(d, b->staging, 3, b->ptab + 10);
  metrics_interior_kernel<<<bgrid(b, (long long)nn), 256, 0, b->stream>>>(d, (const double *const *)(b->ptab + 10),
                                                                           b->ptab + 15, b->aj + bh.off);
  for (int f = 0; f < 6; f++)
    metrics_boundary_kernel<<<bgrid(b, (long long)nn / 4 + 1), 256, 0, b->stream>>>(d, b->ptab + 15, b->aj + bh.off, f);
  const long long all = (long long)(bh.mx + 4) * (bh.my + 4) * (bh.mz + 4);
  ghost_fill_kernel<<<bgrid(b, all), 256, 0, b->stream>>>(d, b->ptab + 15, 10);
  delta2_kernel<<<bgrid(b, d.plane), 256, 0, b->stream>>>(d, b->aj + bh.off, b->delta2 + bh.off);
  BCUDA(b, cudaGetLastError());
  if (b->cfg.precision == CB_MIXED)
    BCUDA(b, launch_mixed_prep(d, (const double *const *)(b->ptab + 15), b->delta2 + bh.off, b->aj + bh.off, b->ptab4,
                               b->ptab + 27, bgrid(b, d.plane), b->stream));
  if (b->coorxy[k])  // x and y kept for the inflow codes that read them
    for (int q = 0; q < 2; q++)
      BCUDA(b, cudaMemcpyAsync(b->coorxy[k] + d.plane * q, b->qb[2][q] + bh.off, sizeof(double) * d.plane,
                               cudaMemcpyDeviceToDevice, b->stream));
  for (int q = 0; q < 3; q++) BCUDA(b, cudaMemsetAsync(b->qb[2][q] + bh.off, 0, sizeof(double) * d.plane, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  bh.have_grid = true;
  if (b->cur == 2) bh.have_state = false;  // the coordinates went through the block's current state buffer
  return CB_OK;
}

int cb_batch_set_nvert(cb_batch *b, int k, const double *nvert) {
  if (check_block(b, k) || !nvert) return CB_E_ARG;
  BlockHost &bh = b->blk[k];
  const size_t nn = (size_t)bh.mx * bh.my * bh.mz;
  if (block_ptab(b, k)) return CB_E_CUDA;
  BCUDA(b, cudaMemcpyAsync(b->staging, nvert, sizeof(double) * nn, cudaMemcpyHostToDevice, b->stream));
  unpack_kernel<<<bgrid(b, (long long)nn), 256, 0, b->stream>>>(bh.dc, b->staging, 1, b->ptab + 25);
  const long long all = (long long)(bh.mx + 4) * (bh.my + 4) * (bh.mz + 4);
  ghost_fill_kernel<<<bgrid(b, all), 256, 0, b->stream>>>(bh.dc, b->ptab + 25, 1);
  BCUDA(b, cudaGetLastError());
  BCUDA(b, cudaStreamSynchronize(b->stream));
  const int q = nvert_codes_exact(nvert, nn);
  bool zero = true;
  for (size_t t = 0; t < nn && zero; t++) zero = nvert[t] == 0.0;
  const bool nv0_was = batch_nv0(b);
  bh.nvz = zero;
  if (q != bh.dc.nvq || batch_nv0(b) != nv0_was) {
    bh.dc.nvq = q;
    if (build_tables(b)) return CB_E_CUDA;  // tables and graphs carry the config and the kernel variant
  }
  return CB_OK;
}

// Face codes of block k.  The reference reads one bcs.dat line per block
// (init.c:556-559) and each block's RungeKutta ends every stage with its own
// FormBCS (solvers.c:246-273, rhs.c:477-1227).  A block with a physical code
// on any face runs that sequence here, on its own arrays, after every stage:
// the RK combine of the boundary shell, the coded faces, the periodic
// directions (code 7 on both faces wraps the block onto itself) and the
// ghost layers -- the kernels and order of the single-block context, so the
// block evolves exactly as it would alone.  Such a block takes no halo-map
// destination; all six codes 7 make it an interface block again.
int cb_batch_set_bctype(cb_batch *b, int k, const int *bctype) {
  if (check_block(b, k) || !bctype) return CB_E_ARG;
  for (int d = 0; d < 3; d++)
    if ((bctype[2 * d] == 7) != (bctype[2 * d + 1] == 7))
      return bfail(b, CB_E_UNSUPPORTED, "a periodic direction needs bctype 7 on both faces");
  bool phys = false;
  for (int f = 0; f < 6; f++) phys = phys || bctype[f] != 7;
  // the k-lo inflow codes 52 and 47 read the node coordinates x, y, which
  // the block keeps from its grid upload
  const bool inflow_xy = bctype[4] == 52 || bctype[4] == 47;
  if (inflow_xy && b->blk[k].have_grid && !b->coorxy[k])
    return bfail(b, CB_E_STATE, "set the inflow codes 52 / 47 before the block's grid");
  if (phys) {
    for (int kind = 0; kind < 2; kind++)
      if (!b->map_dst[kind].empty() && b->map_dst[kind][k])
        return bfail(b, CB_E_ARG, "the block holds halo-map destinations; set face codes before the halo maps");
    if (b->xs.nsend || b->xs.nrecv || b->xw.nsend || b->xw.nrecv)
      return bfail(b, CB_E_UNSUPPORTED, "physical face codes with a cross-process exchange are not built");
  }
  if (block_ib(b, k)) {
    if (!phys) return bfail(b, CB_E_STATE, "a block with immersed-body lists keeps face codes; clear its lists first");
    // its lists' donors were checked against the periodic directions
    for (int d = 0; d < 3; d++)
      if ((bctype[2 * d] == 7) != (b->blk[k].dc.bctype[2 * d] == 7))
        return bfail(b, CB_E_STATE, "a block with immersed-body lists keeps its periodic directions");
  }
  BCUDA(b, cudaStreamSynchronize(b->stream));  // steps in flight read the tables rebuilt below
  BlockHost &bh = b->blk[k];
  if (inflow_xy && !b->coorxy[k]) {
    BCUDA(b, cudaMalloc(&b->coorxy[k], sizeof(double) * 2 * bh.dc.plane));
    BCUDA(b, cudaMemsetAsync(b->coorxy[k], 0, sizeof(double) * 2 * bh.dc.plane, b->stream));
  }
  for (int f = 0; f < 6; f++) bh.dc.bctype[f] = bctype[f];
  bh.phys = phys;
  b->nphys = 0;
  for (const auto &x : b->blk) b->nphys += x.phys ? 1 : 0;
  return build_tables(b);  // the tables carry each block's config; graphs are rebuilt
}

// user->ti of the last completed step (the next step runs ti + 1), read by
// the k-lo inflow code 47; stream-ordered.
int cb_batch_set_time_index(cb_batch *b, int ti) {
  if (!b) return CB_E_ARG;
  BCUDA(b, cudaMemcpyAsync(b->ti_dev, &ti, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  return CB_OK;
}

// ---- immersed bodies: the reference's RungeKutta interpolates every body
// on every block after the block's stages (solvers.c:279-288, one IBMList per
// block and body).  Surfaces are shared by all blocks; lists go to blocks
// with face codes, whose FormBCS(user, 0) follows the interpolation.
static int batch_body(cb_batch *b, int ibi) {
  if (!b) return CB_E_ARG;
  if (ibi < 0 || ibi >= CB_IBM_MAX_BODIES) return bfail(b, CB_E_ARG, "body index out of range");
  return CB_OK;
}

int cb_batch_ibm_set_surface(cb_batch *b, int ibi, int n_v, int n_elmt, const int *nv1, const int *nv2,
                             const int *nv3, const double *nf_x, const double *nf_y, const double *nf_z) {
  if (int e = batch_body(b, ibi)) return e;
  if (n_v < 1 || n_elmt < 1 || !nv1 || !nv2 || !nv3 || !nf_x || !nf_y || !nf_z)
    return bfail(b, CB_E_ARG, "surface needs n_v, n_elmt >= 1 and all arrays");
  BCUDA(b, cudaStreamSynchronize(b->stream));  // graphs in flight may read the old arrays
  for (int k = 0; k < b->nb; k++) ibm_drop_list(b->ibl[(size_t)k * CB_IBM_MAX_BODIES + ibi]);
  IbmBody &sf = b->body[ibi];
  if (sf.surf) cudaFree(sf.surf);
  sf = IbmBody();
  const char *err = "";
  const int rc = ibm_surface_to_device(sf, n_v, n_elmt, nv1, nv2, nv3, nf_x, nf_y, nf_z, b->stream, &err);
  if (rc == CB_E_ARG) return bfail(b, CB_E_ARG, err);
  if (rc) return bfail(b, CB_E_CUDA, "surface upload");
  return build_tables(b);  // lists dropped: the first-stage pressure source changes
}

int cb_batch_ibm_set_velocity(cb_batch *b, int ibi, const double *u, const double *uold) {
  if (int e = batch_body(b, ibi)) return e;
  if (!u || !uold) return CB_E_ARG;
  IbmBody &sf = b->body[ibi];
  if (!sf.surf) return bfail(b, CB_E_STATE, "set the body's surface first");
  BCUDA(b, cudaMemcpyAsync(sf.u, u, sizeof(double) * 3 * sf.n_v, cudaMemcpyHostToDevice, b->stream));
  BCUDA(b, cudaMemcpyAsync(sf.uold, uold, sizeof(double) * 3 * sf.n_v, cudaMemcpyHostToDevice, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  return CB_OK;
}

int cb_batch_ibm_set_list(cb_batch *b, int k, int ibi, int n, const cb_ibm_info *list, const double *coor) {
  if (check_block(b, k)) return CB_E_ARG;
  if (int e = batch_body(b, ibi)) return e;
  if (n < 0 || (n > 0 && (!list || !coor))) return CB_E_ARG;
  if (n > 0 && !b->body[ibi].surf) return bfail(b, CB_E_STATE, "set the body's surface first");
  BlockHost &bh = b->blk[k];
  if (n > 0 && !bh.phys)
    return bfail(b, CB_E_UNSUPPORTED, "immersed bodies need a block with face codes (cb_batch_set_bctype)");
  IbmHostList h;
  const char *err = "";
  if (ibm_build_list(bh.dc, b->cfg.isothermal == 2, b->body[ibi].n_elmt, n, list, coor, h, &err))
    return bfail(b, CB_E_ARG, err);
  BCUDA(b, cudaStreamSynchronize(b->stream));
  IbmBody &l = b->ibl[(size_t)k * CB_IBM_MAX_BODIES + ibi];
  ibm_drop_list(l);
  const bool had = block_ib(b, k);
  if (h.n() > 0) {
    if (!b->ib_arena[k]) {
      const size_t pb = sizeof(double) * 7 * bh.dc.plane;
      BCUDA(b, cudaMalloc(&b->ib_arena[k], pb));
      BCUDA(b, cudaMemsetAsync(b->ib_arena[k], 0, pb, b->stream));
      if (!b->d_ibtab) {
        BCUDA(b, cudaMalloc(&b->d_ibtab, sizeof(double *) * 7 * b->nb));
        BCUDA(b, cudaMemsetAsync(b->d_ibtab, 0, sizeof(double *) * 7 * b->nb, b->stream));
      }
      double *t[7];
      for (int a = 0; a < 7; a++) t[a] = b->ib_arena[k] + bh.dc.plane * a;
      BCUDA(b, cudaMemcpyAsync(b->d_ibtab + 7 * k, t, sizeof(t), cudaMemcpyHostToDevice, b->stream));
    }
    const cudaError_t le = ibm_list_to_device(l, h, b->stream);
    if (le != cudaSuccess) {  // no half-uploaded list stays behind
      ibm_drop_list(l);
      return bfail(b, CB_E_CUDA, std::string("list upload: ") + cudaGetErrorString(le));
    }
    if (!had && bh.have_state) {  // P starts as the EqOfState of the current state
      if (block_ptab(b, k)) return CB_E_CUDA;
      eos_plane_kernel<<<bgrid(b, bh.dc.plane), 256, 0, b->stream>>>(
          bh.dc, (const double *const *)(b->ptab + 5 * b->cur), ib_pl(b, k));
      BCUDA(b, cudaGetLastError());
      BCUDA(b, cudaStreamSynchronize(b->stream));
    }
  }
  return build_tables(b);  // the first-stage pressure source of the block
}

int cb_batch_ibm_set_options(cb_batch *b, int twoD, int wallfunction) {
  if (!b) return CB_E_ARG;
  if (twoD < 0 || twoD > 3) return bfail(b, CB_E_ARG, "twoD must be 0..3");
  if (wallfunction == 1) return bfail(b, CB_E_UNSUPPORTED, "the wall function of -wallfunction 1 is not built");
  if (wallfunction != 0 && wallfunction != 2 && wallfunction != 3)
    return bfail(b, CB_E_ARG, "wallfunction must be 0, 2 or 3");
  b->ibm_twoD = twoD;
  b->ibm_wallfunction = wallfunction;
  destroy_graphs(b);
  return CB_OK;
}

// State of block k (5 per node, AoS) into the CURRENT buffer, ghosts by
// periodic wrap (the halo gather replaces them at every stage).  Resets the
// velocity record of the eddy viscosity, as cb_upload_state does.
int cb_batch_upload_state(cb_batch *b, int k, const double *q) {
  if (check_block(b, k) || !q) return CB_E_ARG;
  BlockHost &bh = b->blk[k];
  const size_t nn = (size_t)bh.mx * bh.my * bh.mz;
  if (b->cfg.precision == CB_MIXED && !b->have_refs) {
    double sp = 0, se = 0, st = 0;
    for (size_t t = 0; t < nn; t++) {
      const double *v = q + 5 * t;
      const double pp = (b->cfg.gamma - 1) * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0]);
      sp += pp; se += v[4]; st += pp / v[0];
    }
    for (auto &x : b->blk) {
      x.dc.p_ref = sp / nn; x.dc.e_ref = se / nn; x.dc.t_ref = st / nn; x.dc.h_ref = x.dc.e_ref + x.dc.p_ref;
    }
    b->have_refs = true;
    if (build_tables(b)) return CB_E_CUDA;
  }
  if (block_ptab(b, k)) return CB_E_CUDA;
  BCUDA(b, cudaMemcpyAsync(b->staging, q, sizeof(double) * 5 * nn, cudaMemcpyHostToDevice, b->stream));
  unpack_kernel<<<bgrid(b, (long long)nn), 256, 0, b->stream>>>(bh.dc, b->staging, 5, b->ptab + 5 * b->cur);
  const long long all = (long long)(bh.mx + 4) * (bh.my + 4) * (bh.mz + 4);
  ghost_fill_kernel<<<bgrid(b, all), 256, 0, b->stream>>>(bh.dc, b->ptab + 5 * b->cur, 5);
  if (block_ib(b, k))  // P starts as the EqOfState of the state, as in a cb_ctx after an upload
    eos_plane_kernel<<<bgrid(b, bh.dc.plane), 256, 0, b->stream>>>(bh.dc, (const double *const *)(b->ptab + 5 * b->cur),
                                                                    ib_pl(b, k));
  BCUDA(b, cudaGetLastError());
  BCUDA(b, cudaMemsetAsync(b->nut + bh.off, 0, sizeof(double) * bh.dc.plane, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  b->uc = -1;
  b->ghosts_dirty = true;
  bh.have_state = true;
  return CB_OK;
}

int cb_batch_download_state(cb_batch *b, int k, double *q) {
  if (check_block(b, k) || !q) return CB_E_ARG;
  BlockHost &bh = b->blk[k];
  const size_t nn = (size_t)bh.mx * bh.my * bh.mz;
  if (block_ptab(b, k)) return CB_E_CUDA;
  pack_kernel<<<bgrid(b, (long long)nn), 256, 0, b->stream>>>(bh.dc, (const double *const *)(b->ptab + 5 * b->cur), 5,
                                                               b->staging);
  BCUDA(b, cudaGetLastError());
  BCUDA(b, cudaMemcpyAsync(q, b->staging, sizeof(double) * 5 * nn, cudaMemcpyDeviceToHost, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  return CB_OK;
}

// CFL time step over every block of the batch: the largest spectral radius
// aj * sum_d (|m_d . u| + c |m_d|) over the fluid interior nodes of all blocks
// (atomicMax into one device word), dt = cfl / lambda_max.
int cb_batch_cfl_dt(cb_batch *b, double cfl, double *dt, double *lambda_max) {
  if (!b || !dt || !(cfl > 0)) return CB_E_ARG;
  for (const auto &bh : b->blk)
    if (!bh.have_grid || !bh.have_state) return bfail(b, CB_E_STATE, "every block needs its grid and state");
  unsigned long long *d = reinterpret_cast<unsigned long long *>(b->staging);  // free between calls
  BCUDA(b, cudaMemsetAsync(d, 0, sizeof(unsigned long long), b->stream));
  for (int k = 0; k < b->nb; k++) {
    const BlockHost &bh = b->blk[k];
    if (block_ptab(b, k)) return CB_E_CUDA;  // stream-ordered after the previous block's launch
    const long long work = (long long)(bh.mx - 2) * (bh.my - 2) * (bh.mz - 2);
    spectral_radius_kernel<<<bgrid(b, work), 256, 0, b->stream>>>(
        bh.dc, (const double *const *)(b->ptab + 5 * b->cur), (const double *const *)(b->ptab + 15), b->aj + bh.off,
        b->nvert + bh.off, d);
    BCUDA(b, cudaGetLastError());
  }
  unsigned long long bits = 0;
  BCUDA(b, cudaMemcpyAsync(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  double lam;
  std::memcpy(&lam, &bits, sizeof(lam));
  if (lambda_max) *lambda_max = lam;
  *dt = lam > 0 ? cfl / lam : 0.0;
  return CB_OK;
}

static bool interior_node(const BlockHost &bh, int i, int j, int k) {
  return i >= 1 && i <= bh.mx - 2 && j >= 1 && j <= bh.my - 2 && k >= 1 && k <= bh.mz - 2;
}

// Metrics of block k as resident (csi, eta, zet: 3 per node; aj: 1), natural AoS.
int cb_batch_get_metrics(cb_batch *b, int k, double *csi, double *eta, double *zet, double *aj) {
  if (check_block(b, k) || !csi || !eta || !zet || !aj) return CB_E_ARG;
  BlockHost &bh = b->blk[k];
  if (!bh.have_grid) return bfail(b, CB_E_STATE, "no grid");
  const size_t nn = (size_t)bh.mx * bh.my * bh.mz;
  if (block_ptab(b, k)) return CB_E_CUDA;
  double *dst[4] = {csi, eta, zet, aj};
  for (int e = 0; e < 4; e++) {
    const int nc = e < 3 ? 3 : 1;
    pack_kernel<<<bgrid(b, (long long)nn), 256, 0, b->stream>>>(bh.dc, (const double *const *)(b->ptab + 15 + 3 * e), nc,
                                                                 b->staging);
    BCUDA(b, cudaGetLastError());
    BCUDA(b, cudaMemcpyAsync(dst[e], b->staging, sizeof(double) * nc * nn, cudaMemcpyDeviceToHost, b->stream));
    BCUDA(b, cudaStreamSynchronize(b->stream));
  }
  return CB_OK;
}

// Halo maps: n entries of 9 ints (dst block, di, dj, dk, src block, si, sj, sk,
// from_stage_input), node indices in -2..m+1.
//   kind CB_HALO_STAGE: applied after every stage; the source is read from the
//     stage output (must then be an interior node) or, with from_stage_input,
//     from the stage input (any node).
//   kind CB_HALO_WRAP: plain wrap (DMGlobalToLocal across blocks), applied to
//     the eddy viscosity every step and once to the uploaded state; the last
//     int is ignored and no source may also be a destination.
// Destinations must be non-interior nodes, each at most once per map.
int cb_batch_set_halo_map(cb_batch *b, int kind, long long n, const int *e) {
  if (!b || n < 0 || (n && !e) || (kind != CB_HALO_STAGE && kind != CB_HALO_WRAP)) return CB_E_ARG;
  std::vector<long long> hd((size_t)n), hs((size_t)n);
  std::vector<unsigned char> hin((size_t)n);
  std::vector<char> dblk((size_t)b->nb, 0);
  for (long long t = 0; t < n; t++) {
    const int *r = e + 9 * t;
    if (r[0] < 0 || r[0] >= b->nb || r[4] < 0 || r[4] >= b->nb) return bfail(b, CB_E_ARG, "halo map: block index");
    const BlockHost &db = b->blk[r[0]], &sb = b->blk[r[4]];
    if (db.phys) return bfail(b, CB_E_ARG, "halo map: destination in a block with a physical face code");
    dblk[r[0]] = 1;
    if (r[1] < -2 || r[1] > db.mx + 1 || r[2] < -2 || r[2] > db.my + 1 || r[3] < -2 || r[3] > db.mz + 1 ||
        r[5] < -2 || r[5] > sb.mx + 1 || r[6] < -2 || r[6] > sb.my + 1 || r[7] < -2 || r[7] > sb.mz + 1)
      return bfail(b, CB_E_ARG, "halo map: node outside the padded box");
    if (interior_node(db, r[1], r[2], r[3])) return bfail(b, CB_E_ARG, "halo map: destination is an interior node");
    const bool fin = kind == CB_HALO_STAGE && r[8] != 0;
    if (kind == CB_HALO_STAGE && !fin && !interior_node(sb, r[5], r[6], r[7]))
      return bfail(b, CB_E_ARG, "halo map: stage-output source is not an interior node");
    hd[t] = db.off + gidx(db.dc, r[1], r[2], r[3]);
    hs[t] = sb.off + gidx(sb.dc, r[5], r[6], r[7]);
    hin[t] = fin ? 1 : 0;
  }
  std::vector<long long> sd(hd);
  std::sort(sd.begin(), sd.end());
  if (std::adjacent_find(sd.begin(), sd.end()) != sd.end()) return bfail(b, CB_E_ARG, "halo map: duplicate destination");
  if (kind == CB_HALO_WRAP)
    for (long long t = 0; t < n; t++)
      if (std::binary_search(sd.begin(), sd.end(), hs[t]))
        return bfail(b, CB_E_ARG, "halo map: wrap source is also a destination");
  long long **pd = kind == CB_HALO_STAGE ? &b->d_hdst : &b->d_wdst;
  long long **ps = kind == CB_HALO_STAGE ? &b->d_hsrc : &b->d_wsrc;
  if (*pd) cudaFree(*pd);
  if (*ps) cudaFree(*ps);
  *pd = *ps = nullptr;
  if (kind == CB_HALO_STAGE) {
    if (b->d_hin) cudaFree(b->d_hin);
    b->d_hin = nullptr;
    b->nhalo = n;
  } else {
    b->nwrap = n;
  }
  if (n) {
    BCUDA(b, cudaMalloc(pd, sizeof(long long) * n));
    BCUDA(b, cudaMalloc(ps, sizeof(long long) * n));
    BCUDA(b, cudaMemcpy(*pd, hd.data(), sizeof(long long) * n, cudaMemcpyHostToDevice));
    BCUDA(b, cudaMemcpy(*ps, hs.data(), sizeof(long long) * n, cudaMemcpyHostToDevice));
    if (kind == CB_HALO_STAGE) {
      BCUDA(b, cudaMalloc(&b->d_hin, n));
      BCUDA(b, cudaMemcpy(b->d_hin, hin.data(), n, cudaMemcpyHostToDevice));
    }
  }
  b->map_dst[kind] = dblk;
  if (kind == CB_HALO_WRAP) b->ghosts_dirty = true;
  destroy_graphs(b);
  return CB_OK;
}

// Self-periodic maps: every block wraps onto itself exactly as the
// single-block periodic path (FormBCS stale copy, rhs.c:1107-1227, then
// DMGlobalToLocal), so each block evolves as it would alone.
int cb_batch_halo_periodic(cb_batch *b) {
  if (!b) return CB_E_ARG;
  std::vector<int> st, wr;
  auto wrapi = [](int x, int m) { return x < 0 ? x + m : (x >= m ? x - m : x); };
  for (int k = 0; k < b->nb; k++) {
    const BlockHost &bh = b->blk[k];
    if (bh.phys) continue;  // its own FormBCS wraps its periodic directions
    for (int kk = -2; kk <= bh.mz + 1; kk++)
      for (int j = -2; j <= bh.my + 1; j++)
        for (int i = -2; i <= bh.mx + 1; i++) {
          if (interior_node(bh, i, j, kk)) continue;
          const int oi = wrapi(i, bh.mx), oj = wrapi(j, bh.my), ok = wrapi(kk, bh.mz);
          // stage map: the device rule of the single-block path (bc_source)
          int si = oi, sj = oj, sk = ok, fin = 0;
          const bool bnd = !interior_node(bh, oi, oj, ok);
          if (bnd) {
            fin = 1;
            if (ok == 0) sk = ok - 2;
            else if (ok == bh.mz - 1) sk = ok + 2;
            else if (oj == 0) sj = oj - 2;
            else if (oj == bh.my - 1) sj = oj + 2;
            else if (oi == 0) si = oi - 2;
            else si = oi + 2;
          }
          const int r[9] = {k, i, j, kk, k, si, sj, sk, fin};
          st.insert(st.end(), r, r + 9);
          // wrap map: ghosts take their owned image; owned nodes keep their value
          const bool ghost = i != oi || j != oj || kk != ok;
          if (ghost) {
            const int w[9] = {k, i, j, kk, k, oi, oj, ok, 0};
            wr.insert(wr.end(), w, w + 9);
          }
        }
  }
  int rc = cb_batch_set_halo_map(b, CB_HALO_STAGE, (long long)(st.size() / 9), st.data());
  if (rc) return rc;
  return cb_batch_set_halo_map(b, CB_HALO_WRAP, (long long)(wr.size() / 9), wr.data());
}

// Applies the wrap map to the current state (after uploads).
static int fill_ghosts(cb_batch *b) {
  if (b->nwrap) {
    for (int q = 0; q < 5; q++)
      plane_gather_kernel<<<bgrid(b, b->nwrap), 256, 0, b->stream>>>(b->d_wdst, b->d_wsrc, b->nwrap, b->qb[b->cur][q]);
    BCUDA(b, cudaGetLastError());
  }
  b->ghosts_dirty = false;
  return CB_OK;
}

static void rk_ab(const cb_batch *b, int s, double *alfa, double *beta) {
  double a[3] = {1., 1 / 4., 2 / 3.}, bb[3] = {1., 3 / 4., 1 / 3.};  // solvers.c:233-234
  if (b->cfg.fluxorder < 3) { a[1] = 1 / 2.; bb[1] = 1 / 2.; }
  *alfa = a[s];
  *beta = bb[s];
}

// One step: eddy viscosity per block, then per stage one stage launch
// (persistent over all blocks, or one per block) and one halo gather.
static int enqueue_nut(cb_batch *b) {
  // Compute_eddy_viscosity_LES per block from the recorded state; the
  // pointer arrays are the q and met members of the block's (uc, uc, uc)
  // table entry in device memory
  if (b->cfg.les == 10) {  // Cs = 0 (les.c:134-137): nu_t stays zero
    BCUDA(b, cudaMemsetAsync(b->nut, 0, sizeof(double) * b->total, b->stream));
    return CB_OK;
  }
  const int u = b->uc < 0 ? 0 : b->uc;
  const bool dyn = batch_dynamic(b->cfg);
  const cb_config &f = b->cfg;
  const DynOpts dopt{f.les, f.max_cs, b->dyn_tf_mult, f.i_homo_filter, f.j_homo_filter, f.k_homo_filter};
  for (int k = 0; k < b->nb; k++) {
    const BlockHost &bh = b->blk[k];
    const long long o = bh.off;
    const long long work = (long long)(bh.mx - 2) * (bh.my - 2) * (bh.mz - 2);
    const char *ent = reinterpret_cast<const char *>(b->d_tables + (size_t)(u * 13) * b->nb + k);
    const double *const *qu = reinterpret_cast<const double *const *>(ent + offsetof(BatchBlock, F) + offsetof(DevFields, q));
    const double *const *mt = reinterpret_cast<const double *const *>(ent + offsetof(BatchBlock, F) + offsetof(DevFields, met));
    // the current state's planes: the q member of the block's (cur, cur, cur) entry
    const char *ecur = reinterpret_cast<const char *>(b->d_tables + (size_t)(b->cur * 13) * b->nb + k);
    const double *const *qc = reinterpret_cast<const double *const *>(ecur + offsetof(BatchBlock, F) + offsetof(DevFields, q));
    double *cs = nullptr;
    if (dyn) {
      // the model on the block's own arrays and ghost layers, as each block of
      // the reference computes it on its own DMDA
      double *const *D = b->d_dynptr + 14 * k;
      double *pl[14];
      for (int a = 0; a < 14; a++) pl[a] = b->dyn_arena + (size_t)b->total * a + o;
      const DynPlanes P{D, pl[9], pl[10], pl[11], pl[12], pl[13]};
      BCUDA(b, dyn_cs_enqueue(bh.dc, dopt, qc, b->uc >= 0 ? qu : nullptr, mt, b->aj + o, b->nvert + o, P, b->sms,
                              b->stream));
      cs = pl[12];
    }
    if (b->cfg.precision == CB_MIXED && !dyn) {  // the mixed form's SGS terms run in FP32
      const float4 *m4[3] = {b->met4[0] + o, b->met4[1] + o, b->met4[2] + o};
      BCUDA(b, launch_eddy_mixed(bh.dc, b->uc >= 0 ? qu : nullptr, m4, bh.nvz ? nullptr : b->nvert + o, b->nut + o,
                                 b->sms, b->stream));
      continue;
    }
    const int ekc = eddy_kchunk(bh.dc, b->sms);
    eddy_viscosity_kernel<<<eddy_grid(bh.dc, ekc), dim3(EDDY_BX, EDDY_BY), 0, b->stream>>>(
        bh.dc, b->uc >= 0 ? qu : nullptr, mt, b->aj + o, b->delta2 + o, bh.nvz ? nullptr : b->nvert + o, b->nut + o, ekc,
        dyn ? qc : nullptr, cs);
  }
  const bool mapped = b->nwrap || b->xw.nsend || b->xw.nrecv;
  if (b->nwrap) plane_gather_kernel<<<bgrid(b, b->nwrap), 256, 0, b->stream>>>(b->d_wdst, b->d_wsrc, b->nwrap, b->nut);
  if (!mapped || b->nphys) {
    // each block's own ghost fill (a block with physical faces always: the
    // single-block context's rule)
    for (int k = 0; k < b->nb; k++) {
      const BlockHost &bh = b->blk[k];
      if (mapped && !bh.phys) continue;
      // a one-entry pointer table: the nut plane of block k sits in the table's nut member
      const char *ent = reinterpret_cast<const char *>(b->d_tables + k);
      double *const *np = reinterpret_cast<double *const *>(ent + offsetof(BatchBlock, F) + offsetof(DevFields, nut));
      ghost_fill_kernel<<<bgrid(b, shell_count(bh.dc)), 256, 0, b->stream>>>(bh.dc, np, 1);
    }
  }
  BCUDA(b, cudaGetLastError());
  return CB_OK;
}

// Ghost layers of the three planes of one sensor pass (arena pointers `ar`,
// per-block pointer tables at offset `toff` of a block's six): the wrap map
// when the batch has one, else each block's own periodic wrap; a block with a
// physical face code always takes its own.
static int sigma_ghosts(cb_batch *b, double *const ar[3], int toff) {
  if (b->nwrap) {
    for (int a = 0; a < 3; a++)
      plane_gather_kernel<<<bgrid(b, b->nwrap), 256, 0, b->stream>>>(b->d_wdst, b->d_wsrc, b->nwrap, ar[a]);
  }
  for (int k = 0; k < b->nb; k++)
    if (!b->nwrap || b->blk[k].phys)
      ghost_fill_kernel<<<bgrid(b, shell_count(b->blk[k].dc)), 256, 0, b->stream>>>(b->blk[k].dc,
                                                                                    b->d_sigptr + 6 * k + toff, 3);
  BCUDA(b, cudaGetLastError());
  return CB_OK;
}

// Hybrid weights of the shock sensor per block from the step's input state
// (formConvectionLES at istage 0, rhs.c:3328-3433): the single-block
// context's three passes, each followed by the ghost fill.  Every block's
// weights come from its own arrays, as each block of the reference computes
// them on its own DMDA.
static int enqueue_sigma(cb_batch *b, int in) {
  const char *tab = reinterpret_cast<const char *>(b->d_tables + (size_t)(in * 13) * b->nb);
  for (int k = 0; k < b->nb; k++) {
    const BlockHost &bh = b->blk[k];
    const char *ent = tab + sizeof(BatchBlock) * k;
    const double *const *q = reinterpret_cast<const double *const *>(ent + offsetof(BatchBlock, F) + offsetof(DevFields, q));
    sigma_sensor_kernel<<<bgrid(b, bh.dc.plane), 256, 0, b->stream>>>(bh.dc, q, b->d_sigptr + 6 * k,
                                                                       block_ib(b, k) ? ib_pl(b, k) : nullptr);
  }
  if (int e = sigma_ghosts(b, b->sig_a, 0)) return e;
  for (int k = 0; k < b->nb; k++)
    sigma_filter_kernel<<<bgrid(b, b->blk[k].dc.plane), 256, 0, b->stream>>>(
        b->blk[k].dc, (const double *const *)(b->d_sigptr + 6 * k), b->d_sigptr + 6 * k + 3);
  if (int e = sigma_ghosts(b, b->sig_b, 3)) return e;
  for (int k = 0; k < b->nb; k++)
    sigma_post_kernel<<<bgrid(b, b->blk[k].dc.plane), 256, 0, b->stream>>>(
        b->blk[k].dc, (const double *const *)(b->d_sigptr + 6 * k + 3), b->d_sigptr + 6 * k);
  return sigma_ghosts(b, b->sig_a, 0);
}

// Stage s of the step that started from buffer `old`: the stage kernel over
// all blocks (persistent or one launch per block), then the local halo gather.
static int enqueue_stage(cb_batch *b, int s, int per_block, int in, int old, int out) {
  const bool les = b->cfg.les != 0, visc = b->cfg.inviscid == 0, mixed = b->cfg.precision == CB_MIXED;
  double alfa, beta;
  rk_ab(b, s, &alfa, &beta);
  const double adt = alfa * b->cfg.dt * b->cfg.st;
  const BatchBlock *tab = b->d_tables + (size_t)(in * 9 + old * 3 + out) * b->nb;
  if (!per_block) {
    BCUDA(b, cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned), b->stream));
    const int ctas = b->sms * (mixed ? 2 : 1);
    BCUDA(b, launch_batched_any(mixed, les, tab, b->d_items, b->nitems, b->d_counter, s, alfa, beta, adt, visc,
                                batch_bits(b), batch_nv0(b), ctas, b->stream));
  } else {
    for (int k = 0; k < b->nb; k++) {
      const BlockHost &bh = b->blk[k];
      const DevFields F = block_fields(b, k, in, old, out);
      const int nk = bh.mz - 2;
      // per-block k-chunk for whole waves of the resident CTAs (the
      // single-block context's rule)
      const int tiles = bh.tiles_x * bh.tiles_y;
      const int slots = b->sms * (mixed ? 2 : 1);
      int kc = nk;
      double best = 1e30;
      for (int cand = 4; cand <= nk; cand++) {
        const long long blocks = (long long)tiles * ((nk + cand - 1) / cand);
        const double cost = (double)((blocks + slots - 1) / slots) * (cand + 1.0);
        if (cost < best) { best = cost; kc = cand; }
      }
      BCUDA(b, launch_stage_any(mixed, les, bh.dc, F, s, alfa, beta, adt, kc, visc, false, batch_bits(b),
                                bh.nvz && !b->cfg.visT, slots, b->stream));
    }
  }
  BCUDA(b, cudaGetLastError());
  if (b->nhalo) {
    DevFields G{};
    for (int q = 0; q < 5; q++) { G.q[q] = b->qb[in][q]; G.qout[q] = b->qb[out][q]; }
    halo_gather_kernel<<<bgrid(b, b->nhalo), 256, 0, b->stream>>>(b->d_hdst, b->d_hsrc, b->d_hin, b->nhalo, G);
    BCUDA(b, cudaGetLastError());
  }
  // blocks with a physical face code: FormBCS with boundary codes on the
  // block's own arrays (rhs.c:477-1227), the single-block context's kernels
  // in its order; no halo-map entry writes into these blocks
  for (int k = 0; k < b->nb && b->nphys; k++) {
    const BlockHost &bh = b->blk[k];
    if (!bh.phys) continue;
    const DevCfg &d = bh.dc;
    const DevFields F = block_fields(b, k, in, old, out);
    const long long shell = shell_count(d);
    bc_combine_kernel<<<bgrid(b, shell), 256, 0, b->stream>>>(d, F, s, alfa, beta, adt);
    const long long face = (long long)std::max(d.mx, d.my) * std::max(d.my, d.mz);
    for (int dir = 0; dir < 3; dir++) bc_face_kernel<<<bgrid(b, face), 256, 0, b->stream>>>(d, F, dir, alfa);
    for (int dir = 0; dir < 3; dir++)
      if (d.bctype[2 * dir] == 7) bc_periodic_dir_kernel<<<bgrid(b, face), 256, 0, b->stream>>>(d, F, dir);
    // the stage output's five plane pointers: the qout member of the block's
    // table entry for this buffer triple (device memory)
    const char *ent = reinterpret_cast<const char *>(tab + k);
    double *const *qo = reinterpret_cast<double *const *>(ent + offsetof(BatchBlock, F) + offsetof(DevFields, qout));
    ghost_fill_kernel<<<bgrid(b, shell), 256, 0, b->stream>>>(d, qo, 5);
    BCUDA(b, cudaGetLastError());
  }
  return CB_OK;
}

// After the stages of a step, on block k with bodies (solvers.c:279-288):
// EqOfState into its pressure plane, five sweeps of ibm_interpolation_advanced
// per body, then FormBCS(user, 0) from snapshots of Q and P (the reference's
// lQ / lP) -- the single-block context's kernels in its order.  `old` is the
// step's input buffer (Qold).
static int enqueue_ib(cb_batch *b, int k, int old) {
  const BlockHost &bh = b->blk[k];
  const DevCfg &d = bh.dc;
  double *pl = ib_pl(b, k), *psnap = b->ib_arena[k] + 5 * d.plane;
  double *const *tab = b->d_ibtab + 7 * k;  // Q snapshot 0..4, P snapshot, carried P
  // the current state's planes: the qout member of the block's (cur, cur, cur) entry
  const char *ent = reinterpret_cast<const char *>(b->d_tables + (size_t)(b->cur * 13) * b->nb + k);
  double *const *qc = reinterpret_cast<double *const *>(ent + offsetof(BatchBlock, F) + offsetof(DevFields, qout));
  eos_plane_kernel<<<bgrid(b, d.plane), 256, 0, b->stream>>>(d, (const double *const *)qc, pl);
  const int slip = (b->cfg.inviscid || b->ibm_wallfunction == 3) ? 1 : 0;  // ibm_iso.c:2721
  const int iso1 = b->cfg.isothermal == 1 ? 1 : 0;
  const int wf2 = b->ibm_wallfunction == 2 ? 1 : 0;
  const bool iso2 = b->cfg.isothermal == 2;
  const double a_sound = sqrt(b->cfg.twall / (b->cfg.ma * b->cfg.ma));  // ibm_iso.c:2768, the host's sqrt
  for (int ibi = 0; ibi < CB_IBM_MAX_BODIES; ibi++) {
    IbmDev dv = b->ibl[(size_t)k * CB_IBM_MAX_BODIES + ibi].dev();
    if (dv.n <= 0) continue;
    const IbmBody &sf = b->body[ibi];
    dv.tri = sf.tri; dv.nf = sf.nf; dv.u = sf.u; dv.uold = sf.uold;
    const int g = bgrid(b, dv.n);
    for (int s = 0; s < IBM_SWEEPS; s++) {
      ibm_interp_kernel<<<g, 256, 0, b->stream>>>(d, (const double *const *)qc, pl, dv, 1, b->ibm_twoD, slip, iso1, wf2,
                                                  iso2 ? b->qb[old][0] + bh.off : nullptr, a_sound);
      if (iso2) {
        ibm_iso2_chain_kernel<<<1, IBM_CHAIN_NT, 0, b->stream>>>(d, dv, s == 0 ? 1 : 0, a_sound);
        ibm_iso2_finish_kernel<<<g, 256, 0, b->stream>>>(d, dv, 1);
      }
      ibm_scatter_kernel<<<g, 256, 0, b->stream>>>(d, qc, pl, dv);
    }
  }
  // FormBCS(user, 0): Q and P within five layers of the faces into the snapshots
  const long long thick = thick_shell_count(d, 5);
  thick_shell_copy_kernel<<<bgrid(b, thick), 256, 0, b->stream>>>(d, 5, (const double *const *)qc, tab, 5);
  thick_shell_copy_kernel<<<bgrid(b, thick), 256, 0, b->stream>>>(d, 5, (const double *const *)(tab + 6), tab + 5, 1);
  DevFields F = block_fields(b, k, b->cur, old, b->cur);
  for (int q = 0; q < 5; q++) F.q[q] = b->ib_arena[k] + d.plane * q;
  F.pin = psnap;
  const long long face = (long long)std::max(d.mx, d.my) * std::max(d.my, d.mz), shell = shell_count(d);
  for (int dir = 0; dir < 3; dir++) bc_face_kernel<<<bgrid(b, face), 256, 0, b->stream>>>(d, F, dir, 0.0);
  for (int dir = 0; dir < 3; dir++)
    if (d.bctype[2 * dir] == 7) {
      bc_periodic_dir_kernel<<<bgrid(b, face), 256, 0, b->stream>>>(d, F, dir);
      bc_periodic_dir_p_kernel<<<bgrid(b, face), 256, 0, b->stream>>>(d, psnap, pl, dir);
    }
  ghost_fill_kernel<<<bgrid(b, shell), 256, 0, b->stream>>>(d, qc, 5);
  ghost_fill_kernel<<<bgrid(b, shell), 256, 0, b->stream>>>(d, tab + 6, 1);
  BCUDA(b, cudaGetLastError());
  return CB_OK;
}

// Buffers of stage s when the step starts from buffer cur0.
static void stage_buffers(int cur0, int s, int *in, int *out) {
  const int A = (cur0 + 1) % 3, B = (cur0 + 2) % 3;
  *out = (s % 2 == 0) ? A : B;
  *in = s == 0 ? cur0 : (((s - 1) % 2 == 0) ? A : B);
}

// One step: eddy viscosity per block, then per stage one stage launch
// (persistent over all blocks, or one per block) and one halo gather.
static int enqueue_batch_step(cb_batch *b, int per_block) {
  // user->ti of the step about to run (the time loop advances it, main.c:887-974)
  for (const auto &bh : b->blk)
    if (bh.dc.bctype[4] == 47) {
      step_index_advance_kernel<<<1, 1, 0, b->stream>>>(b->ti_dev);
      break;
    }
  if (b->cfg.les && !b->cfg.inviscid) {
    int e = enqueue_nut(b);
    if (e) return e;
  }
  const int ns = b->cfg.fluxorder, old = b->cur;
  int in = b->cur, out = b->cur;
  for (int s = 0; s < ns; s++) {
    stage_buffers(old, s, &in, &out);
    if (s == 0 && b->sig_arena) {
      int e = enqueue_sigma(b, in);
      if (e) return e;
    }
    int e = enqueue_stage(b, s, per_block, in, old, out);
    if (e) return e;
    if (!b->cfg.inviscid) b->uc = in;
  }
  b->cur = out;
  for (int k = 0; k < b->nb; k++)
    if (block_ib(b, k)) {
      int e = enqueue_ib(b, k, old);
      if (e) return e;
    }
  return CB_OK;
}

// mode 0: one persistent stage launch over all blocks; 1: one launch per block.
// Steps are captured once per rotation state and replayed as CUDA graphs.
int cb_batch_rk_step(cb_batch *b, int nsteps, int mode) {
  if (!b || nsteps < 0 || (mode != 0 && mode != 1)) return CB_E_ARG;
  for (auto &bh : b->blk)
    if (!bh.have_grid || !bh.have_state) return bfail(b, CB_E_STATE, "every block needs a grid and a state");
  if (!b->nhalo && b->nphys < b->nb)
    return bfail(b, CB_E_STATE, "no halo map (cb_batch_set_halo_map / cb_batch_halo_periodic)");
  if (b->xs.nsend || b->xs.nrecv || b->xw.nsend || b->xw.nrecv)
    return bfail(b, CB_E_STATE, "a batch with a cross-process exchange steps through cb_batch_phase");
  if (b->ghosts_dirty && fill_ghosts(b)) return CB_E_CUDA;
  for (int n = 0; n < nsteps; n++) {
    cudaGraphExec_t &g = b->graphs[mode][b->cur][b->uc + 1];
    if (!g) {
      cudaGraph_t graph;
      const int cur0 = b->cur, uc0 = b->uc;
      BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      int e = enqueue_batch_step(b, mode);
      cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
      if (e) return e;
      if (ce != cudaSuccess) return bfail(b, CB_E_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&g, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return bfail(b, CB_E_CUDA, std::string("instantiate: ") + cudaGetErrorString(ce));
      b->cur = cur0;
      b->uc = uc0;
    }
    BCUDA(b, cudaGraphLaunch(g, b->stream));
    // bookkeeping of the rotation (as enqueue_batch_step)
    const int A = (b->cur + 1) % 3, B = (b->cur + 2) % 3;
    int in = b->cur;
    for (int s = 0; s < b->cfg.fluxorder; s++) {
      if (!b->cfg.inviscid) b->uc = in;
      in = (s % 2 == 0) ? A : B;
    }
    b->cur = in;
  }
  return CB_OK;
}

// Exchange lists of a batch that holds part of a domain whose other parts
// live in other processes.  kind CB_HALO_STAGE: nsend entries of 5 ints
// (block, i, j, k, from_stage_input), nrecv entries of 4 ints (block, i, j, k);
// kind CB_HALO_WRAP: both 4 ints.  d_send / d_recv: caller-owned device
// buffers of 5 doubles per entry.
int cb_batch_set_exchange(cb_batch *b, int kind, long long nsend, const int *send, double *d_send, long long nrecv,
                          const int *recv, double *d_recv) {
  if (!b || (kind != CB_HALO_STAGE && kind != CB_HALO_WRAP) || nsend < 0 || nrecv < 0 || (nsend && (!send || !d_send)) ||
      (nrecv && (!recv || !d_recv)))
    return CB_E_ARG;
  if (b->sig_arena && (nsend || nrecv))
    return bfail(b, CB_E_UNSUPPORTED, "the shock sensor with a cross-process exchange is not built");
  if (b->nphys && (nsend || nrecv))
    return bfail(b, CB_E_UNSUPPORTED, "physical face codes with a cross-process exchange are not built");
  const int sw = kind == CB_HALO_STAGE ? 5 : 4;
  std::vector<long long> hs((size_t)nsend), hd((size_t)nrecv);
  std::vector<unsigned char> hf((size_t)nsend);
  auto in_box = [&](const BlockHost &bh, int i, int j, int k) {
    return i >= -2 && i <= bh.mx + 1 && j >= -2 && j <= bh.my + 1 && k >= -2 && k <= bh.mz + 1;
  };
  for (long long t = 0; t < nsend; t++) {
    const int *r = send + sw * t;
    if (r[0] < 0 || r[0] >= b->nb) return bfail(b, CB_E_ARG, "exchange: block index");
    const BlockHost &bh = b->blk[r[0]];
    if (!in_box(bh, r[1], r[2], r[3])) return bfail(b, CB_E_ARG, "exchange: node outside the padded box");
    const bool fin = kind == CB_HALO_STAGE && r[4] != 0;
    if (kind == CB_HALO_STAGE && !fin && !interior_node(bh, r[1], r[2], r[3]))
      return bfail(b, CB_E_ARG, "exchange: stage-output source is not an interior node");
    hs[t] = bh.off + gidx(bh.dc, r[1], r[2], r[3]);
    hf[t] = fin ? 1 : 0;
  }
  for (long long t = 0; t < nrecv; t++) {
    const int *r = recv + 4 * t;
    if (r[0] < 0 || r[0] >= b->nb) return bfail(b, CB_E_ARG, "exchange: block index");
    const BlockHost &bh = b->blk[r[0]];
    if (!in_box(bh, r[1], r[2], r[3])) return bfail(b, CB_E_ARG, "exchange: node outside the padded box");
    if (interior_node(bh, r[1], r[2], r[3])) return bfail(b, CB_E_ARG, "exchange: destination is an interior node");
    hd[t] = bh.off + gidx(bh.dc, r[1], r[2], r[3]);
  }
  std::vector<long long> sd(hd);
  std::sort(sd.begin(), sd.end());
  if (std::adjacent_find(sd.begin(), sd.end()) != sd.end()) return bfail(b, CB_E_ARG, "exchange: duplicate destination");
  Xchg &x = kind == CB_HALO_STAGE ? b->xs : b->xw;
  if (x.d_src) cudaFree(x.d_src);
  if (x.d_dst) cudaFree(x.d_dst);
  if (x.d_fin) cudaFree(x.d_fin);
  x = Xchg();
  x.nsend = nsend;
  x.nrecv = nrecv;
  x.d_send = d_send;
  x.d_recv = d_recv;
  if (nsend) {
    BCUDA(b, cudaMalloc(&x.d_src, sizeof(long long) * nsend));
    BCUDA(b, cudaMemcpy(x.d_src, hs.data(), sizeof(long long) * nsend, cudaMemcpyHostToDevice));
    if (kind == CB_HALO_STAGE) {
      BCUDA(b, cudaMalloc(&x.d_fin, nsend));
      BCUDA(b, cudaMemcpy(x.d_fin, hf.data(), nsend, cudaMemcpyHostToDevice));
    }
  }
  if (nrecv) {
    BCUDA(b, cudaMalloc(&x.d_dst, sizeof(long long) * nrecv));
    BCUDA(b, cudaMemcpy(x.d_dst, hd.data(), sizeof(long long) * nrecv, cudaMemcpyHostToDevice));
  }
  destroy_graphs(b);
  return CB_OK;
}

static FieldSet field_set(const double *const *in, const double *const *out, int nf) {
  FieldSet fs{};
  for (int f = 0; f < nf; f++) { fs.in[f] = in ? in[f] : nullptr; fs.out[f] = out[f]; }
  return fs;
}

// Enqueues one phase of a step with a cross-process exchange and packs what
// this process sends; the caller then exchanges the buffers (all on the
// batch's stream) and calls cb_batch_phase_unpack.  Phases:
//   CB_PHASE_STATE  once after the uploads: wrap map on the state, pack of the
//                   state's wrap values (5 per entry)
//   CB_PHASE_NUT    each step with LES: eddy viscosity, wrap map, pack (1 per entry)
//   CB_PHASE_STAGE  stage `stage` (0, 1, ... in order): stage kernel, stage
//                   map, pack of the stage values (5 per entry)
int cb_batch_phase(cb_batch *b, int phase, int stage, int mode) {
  if (!b || (mode != 0 && mode != 1)) return CB_E_ARG;
  for (int k = 0; k < b->nb; k++)
    if (block_ib(b, k)) return bfail(b, CB_E_UNSUPPORTED, "immersed bodies with the phase API are not built");
  if (b->sig_arena) return bfail(b, CB_E_UNSUPPORTED, "the shock sensor with a cross-process exchange is not built");
  for (auto &bh : b->blk)
    if (!bh.have_grid || !bh.have_state) return bfail(b, CB_E_STATE, "every block needs a grid and a state");
  if (phase == CB_PHASE_STATE) {
    if (fill_ghosts(b)) return CB_E_CUDA;
    if (b->xw.nsend) {
      const double *qs[5];
      for (int q = 0; q < 5; q++) qs[q] = b->qb[b->cur][q];
      xpack_kernel<<<bgrid(b, b->xw.nsend), 256, 0, b->stream>>>(b->xw.d_src, nullptr, b->xw.nsend, 5,
                                                                  field_set(nullptr, qs, 5), b->xw.d_send);
    }
  } else if (phase == CB_PHASE_NUT) {
    if (!(b->cfg.les && !b->cfg.inviscid)) return bfail(b, CB_E_STATE, "no eddy viscosity without les and viscosity");
    if (b->ghosts_dirty) return bfail(b, CB_E_STATE, "run CB_PHASE_STATE after uploads");
    int e = enqueue_nut(b);
    if (e) return e;
    if (b->xw.nsend) {
      const double *ns[1] = {b->nut};
      xpack_kernel<<<bgrid(b, b->xw.nsend), 256, 0, b->stream>>>(b->xw.d_src, nullptr, b->xw.nsend, 1,
                                                                  field_set(nullptr, ns, 1), b->xw.d_send);
    }
  } else if (phase == CB_PHASE_STAGE) {
    if (b->ghosts_dirty) return bfail(b, CB_E_STATE, "run CB_PHASE_STATE after uploads");
    if (stage != b->xnext || stage < 0 || stage >= b->cfg.fluxorder) return bfail(b, CB_E_STATE, "stages must run in order");
    if (stage == 0) b->xcur0 = b->cur;
    int in, out;
    stage_buffers(b->xcur0, stage, &in, &out);
    int e = enqueue_stage(b, stage, mode, in, b->xcur0, out);
    if (e) return e;
    if (b->xs.nsend) {
      const double *qi[5], *qo[5];
      for (int q = 0; q < 5; q++) { qi[q] = b->qb[in][q]; qo[q] = b->qb[out][q]; }
      xpack_kernel<<<bgrid(b, b->xs.nsend), 256, 0, b->stream>>>(b->xs.d_src, b->xs.d_fin, b->xs.nsend, 5,
                                                                  field_set(qi, qo, 5), b->xs.d_send);
    }
    b->xin = in;
    b->xout = out;
  } else {
    return CB_E_ARG;
  }
  BCUDA(b, cudaGetLastError());
  return CB_OK;
}

int cb_batch_phase_unpack(cb_batch *b, int phase) {
  if (!b) return CB_E_ARG;
  OutSet os{};
  int nf = 5;
  const Xchg *x = &b->xw;
  if (phase == CB_PHASE_STATE) {
    for (int q = 0; q < 5; q++) os.a[q] = b->qb[b->cur][q];
  } else if (phase == CB_PHASE_NUT) {
    os.a[0] = b->nut;
    nf = 1;
  } else if (phase == CB_PHASE_STAGE) {
    if (b->xout < 0) return bfail(b, CB_E_STATE, "no stage to unpack");
    for (int q = 0; q < 5; q++) os.a[q] = b->qb[b->xout][q];
    x = &b->xs;
  } else {
    return CB_E_ARG;
  }
  if (x->nrecv)
    xunpack_kernel<<<bgrid(b, x->nrecv), 256, 0, b->stream>>>(x->d_dst, x->nrecv, nf, os, x->d_recv);
  BCUDA(b, cudaGetLastError());
  if (phase == CB_PHASE_STAGE) {
    if (!b->cfg.inviscid) b->uc = b->xin;
    const int s = b->xnext;
    b->xnext = s + 1;
    if (b->xnext == b->cfg.fluxorder) {  // step complete
      b->cur = b->xout;
      b->xnext = 0;
      b->xcur0 = -1;
    }
    b->xout = -1;
  }
  return CB_OK;
}

int cb_batch_sync(cb_batch *b) {
  if (!b) return CB_E_ARG;
  BCUDA(b, cudaStreamSynchronize(b->stream));
  unsigned st = 0;
  BCUDA(b, cudaMemcpy(&st, b->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (st) {
    BCUDA(b, cudaMemset(b->status, 0, sizeof(unsigned)));
    return bfail(b, CB_E_NONFINITE, "device status: non-finite state or rho/p <= 0");
  }
  return CB_OK;
}

// Autotuner: times one stage launch of the persistent form for each candidate
// k-chunk (largest-first item list rebuilt each time) and keeps the fastest.
// The state is not advanced: the timed launches write a scratch buffer pair.
int cb_batch_autotune(cb_batch *b, int *best_kchunk, double *best_ms) {
  if (!b) return CB_E_ARG;
  for (auto &bh : b->blk)
    if (!bh.have_grid || !bh.have_state) return bfail(b, CB_E_STATE, "every block needs a grid and a state");
  const int cands[] = {6, 8, 12, 16, 24, 32, 48};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const bool les = b->cfg.les != 0, visc = b->cfg.inviscid == 0, mixed = b->cfg.precision == CB_MIXED;
  int best = b->kchunk;
  double bms = 1e30;
  // the timed launches write a buffer that holds neither the state nor the
  // recorded velocity field of the next eddy-viscosity evaluation
  const int in = b->cur;
  int out = (b->cur + 1) % 3;
  if (out == b->uc) out = (b->cur + 2) % 3;
  for (int kc : cands) {
    b->kchunk = kc;
    if (build_tables(b)) return CB_E_CUDA;
    const BatchBlock *tab = b->d_tables + (size_t)(in * 9 + in * 3 + out) * b->nb;
    float tot = 0.f;
    for (int rep = 0; rep < 3; rep++) {
      cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned), b->stream);
      cudaEventRecord(e0, b->stream);
      const int ctas = b->sms * (mixed ? 2 : 1);
      launch_batched_any(mixed, les, tab, b->d_items, b->nitems, b->d_counter, 0, 1.0, 1.0, 0.0, visc,
                         batch_bits(b), batch_nv0(b), ctas, b->stream);
      cudaEventRecord(e1, b->stream);
      BCUDA(b, cudaEventSynchronize(e1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep) tot += ms;  // first launch warms caches
    }
    const double avg = tot / 2.0;
    if (avg < bms) { bms = avg; best = kc; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->kchunk = best;
  if (build_tables(b)) return CB_E_CUDA;
  if (best_kchunk) *best_kchunk = best;
  if (best_ms) *best_ms = bms;
  return CB_OK;
}

}  // extern "C"
