// Dynamic Smagorinsky model (Compute_Smagorinsky_Constant_1 with a dynamic
// -les, les.c:151-1472, the 3-D box test filter): Germano's identity with a
// 3x3x3 test filter, the least-squares ratio LM / MM averaged over 27 nodes,
// clipping, and a 1/aj-weighted 27-node mean of the coefficient.  With -les 3
// or a homogeneous filter LM / MM are taken node by node, the plane / line /
// box means of -i/-j/-k_homo_filter replace them, and the final mean is
// skipped.  Runs once per step before the eddy viscosity, all in FP64 on the
// ghosted current state.
//
// The reference overwrites lUcat in place in its first loop (les.c:234-238):
// a node's velocity becomes rhoU/rho of the current state once the loop has
// reached it (interior nodes with nvert <= 1.1), so that loop's central
// differences see the new value at the i-1, j-1, k-1 neighbours and the value
// of the last CalcUCat (the state `qu`) at the +1 neighbours; everything
// after it sees the new value at every such node.  dyn_u reproduces that.
#pragma once
#include "cb_common.cuh"

namespace cb {

constexpr double DYN_EPS = 0.000001;  // les.c:8

__device__ __forceinline__ bool dyn_interior(const DevCfg &c, int i, int j, int k) {
  return i >= 1 && i <= c.mx - 2 && j >= 1 && j <= c.my - 2 && k >= 1 && k <= c.mz - 2;
}

__device__ __forceinline__ double dyn_u(const DevCfg &c, const double *const *q, const double *const *qu,
                                        const double *nvert, int a, int i, int j, int k, bool reached) {
  const long long m = gidx(c, i, j, k);
  if (reached && dyn_interior(c, i, j, k) && nvert[m] <= 1.1) return q[1 + a][m] / q[0][m];  // les.c:255, x kept
  if (a == 0 && c.twod == 1) return 0.0;  // the last CalcUCat's x with -twoD 1 (rhs.c:1349)
  return qu ? qu[1 + a][m] / qu[0][m] : 0.0;
}

__device__ __forceinline__ void dyn_node(const DevCfg &c, long long t, int &i, int &j, int &k) {
  const unsigned u = (unsigned)t, px = (unsigned)c.px, py = (unsigned)c.py;
  const unsigned row = u / px;
  i = (int)(u - row * px) - 2;
  j = (int)(row % py) - 2;
  k = (int)(row / py) - 2;
}

// (1) velocity gradients (du/dx .. dw/dz) and |S| at interior nodes with
// nvert <= 1.1 (les.c:234-284); zero on every other node of the padded box.
static __global__ void dyn_grad_kernel(const DevCfg c, const double *const *q, const double *const *qu,
                                       const double *const *met, const double *aj, const double *nvert,
                                       double *const *A, double *Sabs) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < c.plane; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    dyn_node(c, t, i, j, k);
    double g[3][3] = {{0., 0., 0.}, {0., 0., 0.}, {0., 0., 0.}};
    double sabs = 0.;
    if (i <= c.mx + 1 && j <= c.my + 1 && dyn_interior(c, i, j, k) && nvert[t] <= 1.1) {
      double d[3][3];
#pragma unroll
      for (int a = 0; a < 3; a++) {
        d[a][0] = (dyn_u(c, q, qu, nvert, a, i + 1, j, k, false) - dyn_u(c, q, qu, nvert, a, i - 1, j, k, true)) * 0.5;
        d[a][1] = (dyn_u(c, q, qu, nvert, a, i, j + 1, k, false) - dyn_u(c, q, qu, nvert, a, i, j - 1, k, true)) * 0.5;
        d[a][2] = (dyn_u(c, q, qu, nvert, a, i, j, k + 1, false) - dyn_u(c, q, qu, nvert, a, i, j, k - 1, true)) * 0.5;
      }
      const double ajc = aj[t];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int x = 0; x < 3; x++)
          g[a][x] = (d[a][0] * met[0 * 3 + x][t] + d[a][1] * met[1 * 3 + x][t] + d[a][2] * met[2 * 3 + x][t]) * ajc;
      const double Sdd = 2. / 3. * (g[0][0] + g[1][1] + g[2][2]);
      const double Sxx = 0.5 * (g[0][0] + g[0][0]) - Sdd, Sxy = 0.5 * (g[0][1] + g[1][0]), Sxz = 0.5 * (g[0][2] + g[2][0]);
      const double Syy = 0.5 * (g[1][1] + g[1][1]) - Sdd, Syz = 0.5 * (g[1][2] + g[2][1]);
      const double Szz = 0.5 * (g[2][2] + g[2][2]) - Sdd;
      sabs = sqrt(2.0 * (Sxx * Sxx + Sxy * Sxy + Sxz * Sxz + Sxy * Sxy + Syy * Syy + Syz * Syz + Sxz * Sxz + Syz * Syz +
                         Szz * Szz));
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int x = 0; x < 3; x++) A[3 * a + x][t] = g[a][x];
    Sabs[t] = sabs;
  }
}

// Boundary nodes of the periodic directions from two nodes across, over the
// interior ranges of the other two directions (les.c:287-353, 1217-1271);
// the three faces' node sets are disjoint.
static __global__ void dyn_copy_kernel(const DevCfg c, double *const *f, int nplanes) {
  const long long ni = (long long)(c.my - 2) * (c.mz - 2), nj = (long long)(c.mx - 2) * (c.mz - 2),
                  nk = (long long)(c.mx - 2) * (c.my - 2);
  const long long total = ni + nj + nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int dir;
    long long r = t;
    int a, b;
    if (r < ni) { dir = 0; a = 1 + (int)(r % (c.my - 2)); b = 1 + (int)(r / (c.my - 2)); }
    else if ((r -= ni) < nj) { dir = 1; a = 1 + (int)(r % (c.mx - 2)); b = 1 + (int)(r / (c.mx - 2)); }
    else { r -= nj; dir = 2; a = 1 + (int)(r % (c.mx - 2)); b = 1 + (int)(r / (c.mx - 2)); }
    if (c.bctype[2 * dir] != 7 && c.bctype[2 * dir + 1] != 7) continue;
    long long lo, hi;
    if (dir == 0) { lo = gidx(c, 0, a, b); hi = gidx(c, c.mx - 1, a, b); }
    else if (dir == 1) { lo = gidx(c, a, 0, b); hi = gidx(c, a, c.my - 1, b); }
    else { lo = gidx(c, a, b, 0); hi = gidx(c, a, b, c.mz - 1); }
    const long long s = gstride(c, dir);
    for (int p = 0; p < nplanes; p++) {
      f[p][lo] = f[p][lo - 2 * s];
      f[p][hi] = f[p][hi + 2 * s];
    }
  }
}

// (2) LM and MM of Germano's identity at interior nodes with nvert <= 1.1
// (les.c:442-792): the test-filtered products of the 27 nodes around, with
// weights 1/(|r|+1)/(|q|+1)/(|p|+1), accumulated in the reference's k, j, i
// order (the caller zeroes every other node).  The pressure-velocity terms
// (beta) feed nothing downstream and are not formed.  A block owns a
// DYN_BX x DYN_BY column of interior nodes and marches along k through a
// chunk of planes, keeping three planes (k-1, k, k+1, with a one-node halo in
// i and j) of the per-node inputs in shared memory -- velocity as lUcat holds
// it, rho, rhoU, rhoV, rhoW, the six distinct strain components and |S| -- so
// each input is formed once per node instead of once per neighbour.
constexpr int DYN_BX = 32, DYN_BY = 6, DYN_PX = DYN_BX + 2, DYN_PN = DYN_PX * (DYN_BY + 2), DYN_NF = 14;
constexpr size_t DYN_LM_SMEM = sizeof(double) * 3 * DYN_NF * DYN_PN;
static __global__ void __launch_bounds__(DYN_BX *DYN_BY)
    dyn_lm_tiled_kernel(const DevCfg c, const double *const *q, const double *const *qu, const double *aj,
                        const double *nvert, const double *const *A, const double *Sabs, double *LM, double *MM,
                        int kchunk, double tf_mult) {
  extern __shared__ double dsm[];  // [slot][field][node]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * DYN_BX + tx;
  const int i0 = 1 + blockIdx.x * DYN_BX, j0 = 1 + blockIdx.y * DYN_BY;
  const int kb = 1 + blockIdx.z * kchunk, ke = min(c.mz - 1, kb + kchunk);
  const int i = i0 + tx, j = j0 + ty;
  const bool act = i <= c.mx - 2 && j <= c.my - 2;
  auto load = [&](int kk, int s) {
    double *base = dsm + (size_t)s * DYN_NF * DYN_PN;
    for (int e = tid; e < DYN_PN; e += DYN_BX * DYN_BY) {
      const int lx = e % DYN_PX, ly = e / DYN_PX;
      const int xi = i0 - 1 + lx, yj = j0 - 1 + ly;
      double v[DYN_NF];
#pragma unroll
      for (int f = 0; f < DYN_NF; f++) v[f] = 0.;
      if (xi <= c.mx - 1 && yj <= c.my - 1) {
        const long long m = gidx(c, xi, yj, kk);
        v[0] = dyn_u(c, q, qu, nvert, 0, xi, yj, kk, true);
        v[1] = dyn_u(c, q, qu, nvert, 1, xi, yj, kk, true);
        v[2] = dyn_u(c, q, qu, nvert, 2, xi, yj, kk, true);
        v[3] = q[0][m]; v[4] = q[1][m]; v[5] = q[2][m]; v[6] = q[3][m];
        v[7] = 0.5 * (A[0][m] + A[0][m]); v[8] = 0.5 * (A[1][m] + A[3][m]); v[9] = 0.5 * (A[2][m] + A[6][m]);
        v[10] = 0.5 * (A[4][m] + A[4][m]); v[11] = 0.5 * (A[5][m] + A[7][m]); v[12] = 0.5 * (A[8][m] + A[8][m]);
        v[13] = Sabs[m];
      }
#pragma unroll
      for (int f = 0; f < DYN_NF; f++) base[f * DYN_PN + e] = v[f];
    }
  };
  load(kb - 1, (kb - 1) % 3);
  load(kb, kb % 3);
  for (int k = kb; k < ke; k++) {
    load(k + 1, (k + 1) % 3);
    __syncthreads();
    if (act) {
      const long long n = gidx(c, i, j, k);
      double lm = 0., mm = 0.;
      if (nvert[n] <= 1.1) {
        double f[22];
#pragma unroll
        for (int x = 0; x < 22; x++) f[x] = 0.;
        double ws = 0.;
        double Sc[6];
        for (int R = 0; R < 3; R++) {
          const double *pl = dsm + (size_t)((k + R - 1) % 3) * DYN_NF * DYN_PN;
          for (int Q = 0; Q < 3; Q++)
#pragma unroll
            for (int P = 0; P < 3; P++) {
              const int e = (ty + Q) * DYN_PX + tx + P;
              const double w = 1. / (fabs(R - 1.0) + 1) * 1. / (fabs(Q - 1.0) + 1) * 1. / (fabs(P - 1.0) + 1);
              const double u = pl[0 * DYN_PN + e], v = pl[1 * DYN_PN + e], ww = pl[2 * DYN_PN + e];
              const double rho = pl[3 * DYN_PN + e], ru = pl[4 * DYN_PN + e], rv = pl[5 * DYN_PN + e],
                           rw = pl[6 * DYN_PN + e];
              const double sm = pl[13 * DYN_PN + e];
              const double val[10] = {rho, ru, rv, rw, ru * u, ru * v, ru * ww, rv * v, rv * ww, rw * ww};
#pragma unroll
              for (int x = 0; x < 10; x++) f[x] += w * val[x];
#pragma unroll
              for (int x = 0; x < 6; x++) {
                const double S = pl[(7 + x) * DYN_PN + e];
                f[10 + x] += w * S;
                f[16 + x] += w * (S * sm * rho);
                if (R == 1 && Q == 1 && P == 1) Sc[x] = S;
              }
              ws += w;
            }
        }
        // the weights sum to 8 exactly (powers of two), so dividing by the
        // sum is the exact scaling by its reciprocal
        const double rws = 1.0 / ws;
        const double _rho = f[0] * rws, _rhou = f[1] * rws, _rhov = f[2] * rws, _rhow = f[3] * rws;
        const int sym[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
        const int prod[3][3] = {{4, 5, 6}, {5, 7, 8}, {6, 8, 9}};
        const double fr[3] = {_rhou, _rhov, _rhow};
        double Lij[3][3], Sh[3][3], SSh[3][3], Sx[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int b = 0; b < 3; b++) {
            Lij[a][b] = f[prod[a][b]] * rws - fr[a] * fr[b] / _rho;
            Sh[a][b] = f[10 + sym[a][b]] * rws;
            SSh[a][b] = f[16 + sym[a][b]] * rws;
            Sx[a][b] = Sc[sym[a][b]];
          }
        // pow(x, 2.) of the reference = x * x, the correctly rounded square
        double S_hat = 0;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int b = 0; b < 3; b++) S_hat += Sh[a][b] * Sh[a][b];
        S_hat = sqrt(2 * S_hat);
        const double filter = pow(1. / aj[n], 1. / 3.);
        const double test_filter = tf_mult * filter;  // 2, or 5^(1/3) with -testfilter_ik (les.c:598-601)
        const double tf2 = test_filter * test_filter, f2 = filter * filter;
        double L_cat = 0.0, M_cat = 0.0;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int b = 0; b < 3; b++) {
            M_cat += -2.0 * _rho * tf2 * S_hat * (Sh[a][b] * Sx[a][b] - 0.33 * Sh[a][a] * Sx[b][b]) +
                     2.0 * f2 * (SSh[a][b] * Sx[a][b] - 0.33 * SSh[a][a] * Sx[b][b]);
            L_cat += Lij[a][b] * Sx[a][b] - 0.33 * Sx[a][a] * Lij[b][b];
          }
        lm = L_cat;
        mm = M_cat;
      }
      LM[n] = lm;
      MM[n] = mm;
    }
    __syncthreads();  // the slot of plane k-1 is refilled next
  }
}

// (3) Cs from the 27-node means of LM and MM at interior nodes
// (les.c:905-925), or from LM / MM of the node itself (pointwise: -les 3 or a
// homogeneous filter), then, with clip, the clipping of every owned node
// (les.c:1124-1137, whose face tests compare !bctype with 7 and never hold);
// boundary nodes keep their previous value through it.
__device__ __forceinline__ double dyn_clip(double v, double nv, double max_cs) {
  if (nv > 1.1 && nv < 7.) return 0.0;
  if (nv > 0.1 && nv < 1.1) v = (0.01 < v) ? v : 0.01;
  const double tt = (v < 0.000) ? 0.000 : v;
  return (tt < max_cs) ? tt : max_cs;
}

static __global__ void dyn_cs_kernel(const DevCfg c, const double *nvert, const double *LM, const double *MM,
                                     double *cs, double max_cs, int pointwise, int clip) {
  const long long total = (long long)c.mx * c.my * c.mz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const unsigned u = (unsigned)t;
    const int i = (int)(u % (unsigned)c.mx), j = (int)((u / (unsigned)c.mx) % (unsigned)c.my),
              k = (int)(u / ((unsigned)c.mx * (unsigned)c.my));
    const long long n = gidx(c, i, j, k);
    const double nv = nvert[n];
    double v = cs[n];
    if (dyn_interior(c, i, j, k)) {
      if (nv > 1.1) {
        v = 0;
      } else {
        double lm = 0.0, mm = 0.0;
        if (pointwise) {
          lm = LM[n];
          mm = MM[n];
        } else {
          for (int R = 0; R < 3; R++)
            for (int Q = 0; Q < 3; Q++)
              for (int P = 0; P < 3; P++) {
                const long long m = gidx(c, i + P - 1, j + Q - 1, k + R - 1);
                lm += LM[m] / 27.0;
                mm += MM[m] / 27.0;
              }
        }
        const double C = lm / (mm + DYN_EPS);
        v = (C < 0.0001) ? 0.0001 : C;
      }
    }
    cs[n] = clip ? dyn_clip(v, nv, max_cs) : v;
  }
}

// Homogeneous averages of LM and MM (les.c:934-1115).  The reference sums in
// k, j, i loop order on one rank; the i-line means here keep that order, the
// plane and box sums are deterministic tree reductions (the same result on
// every run, within a few ulps of the sequential sum).
constexpr int DYN_RED = 256;

// tree sum of one value per thread of a DYN_RED-thread block; every thread
// gets the total
__device__ __forceinline__ double dyn_block_sum(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int x = 0; x < DYN_RED / 32; x++) t += red[x];
  return t;
}

// -i_homo_filter with -k_homo_filter: one block per j plane sums LM, MM and
// the count over its fluid (nvert < 0.1) interior nodes, then every interior
// node of the plane gets 0.5 <LM> / (<MM> + eps)  (les.c:934-980).
static __global__ void __launch_bounds__(DYN_RED) dyn_homo_plane_kernel(const DevCfg c, const double *nvert,
                                                                        const double *LM, const double *MM,
                                                                        double *cs) {
  __shared__ double red[DYN_RED / 32];
  const int j = 1 + blockIdx.x;
  const int nx = c.mx - 2, nz = c.mz - 2;
  const int cnt_all = nx * nz;
  double lm = 0.0, mm = 0.0, cn = 0.0;
  for (int t = threadIdx.x; t < cnt_all; t += DYN_RED) {
    const int i = 1 + t % nx, k = 1 + t / nx;
    const long long n = gidx(c, i, j, k);
    if (nvert[n] < 0.1) { lm += LM[n]; mm += MM[n]; cn += 1.0; }
  }
  lm = dyn_block_sum(lm, red);
  mm = dyn_block_sum(mm, red);
  cn = dyn_block_sum(cn, red);
  if (cn > 0.0) { lm /= cn; mm /= cn; }
  const double v = 0.5 * lm / (mm + DYN_EPS);
  for (int t = threadIdx.x; t < cnt_all; t += DYN_RED) {
    const int i = 1 + t % nx, k = 1 + t / nx;
    cs[gidx(c, i, j, k)] = v;
  }
}

// -i_homo_filter without -k_homo_filter: one thread per (k, j) line sums
// along i in the reference's order; fluid interior nodes of the line get
// 0.5 <LM> / (<MM> + eps)  (les.c:984-1081).
static __global__ void dyn_homo_line_kernel(const DevCfg c, const double *nvert, const double *LM, const double *MM,
                                            double *cs) {
  const int ny = c.my - 2, nz = c.mz - 2;
  const int lines = ny * nz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < lines; t += gridDim.x * blockDim.x) {
    const int j = 1 + t % ny, k = 1 + t / ny;
    const long long row = gidx(c, 0, j, k);
    double lm = 0.0, mm = 0.0;
    int cnt = 0;
    for (int i = 1; i < c.mx - 1; i++)
      if (nvert[row + i] < 0.1) { lm += LM[row + i]; mm += MM[row + i]; cnt++; }
    if (cnt > 0) { lm /= (double)cnt; mm /= (double)cnt; }
    const double v = 0.5 * lm / (mm + DYN_EPS);
    for (int i = 1; i < c.mx - 1; i++)
      if (nvert[row + i] < 0.1) cs[row + i] = v;
  }
}

// -i/-j/-k_homo_filter together, first pass: per-block sums of LM and MM over
// every interior node (no mask) into part[2 * block] (les.c:1087-1101).
static __global__ void __launch_bounds__(DYN_RED) dyn_homo_box_partial_kernel(const DevCfg c, const double *LM,
                                                                              const double *MM, double *part) {
  __shared__ double red[DYN_RED / 32];
  const long long nx = c.mx - 2, ny = c.my - 2, total = nx * ny * (c.mz - 2);
  double lm = 0.0, mm = 0.0;
  for (long long t = blockIdx.x * (long long)DYN_RED + threadIdx.x; t < total; t += (long long)gridDim.x * DYN_RED) {
    const int i = 1 + (int)(t % nx), j = 1 + (int)((t / nx) % ny), k = 1 + (int)(t / (nx * ny));
    const long long n = gidx(c, i, j, k);
    lm += LM[n];
    mm += MM[n];
  }
  lm = dyn_block_sum(lm, red);
  mm = dyn_block_sum(mm, red);
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = lm; part[2 * blockIdx.x + 1] = mm; }
}

// second pass (one block): the box value sum LM / sum MM into part[2 * nparts]
static __global__ void __launch_bounds__(DYN_RED) dyn_homo_box_final_kernel(double *part, int nparts) {
  __shared__ double red[DYN_RED / 32];
  double lm = 0.0, mm = 0.0;
  for (int b = threadIdx.x; b < nparts; b += DYN_RED) { lm += part[2 * b]; mm += part[2 * b + 1]; }
  lm = dyn_block_sum(lm, red);
  mm = dyn_block_sum(mm, red);
  if (threadIdx.x == 0) part[2 * nparts] = lm / mm;
}

// The clipping of every owned node (les.c:1124-1137) after the homogeneous
// averages; with box, every owned node first takes the box value.
static __global__ void dyn_clip_kernel(const DevCfg c, const double *nvert, double *cs, double max_cs,
                                       const double *box) {
  const long long total = (long long)c.mx * c.my * c.mz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const unsigned u = (unsigned)t;
    const int i = (int)(u % (unsigned)c.mx), j = (int)((u / (unsigned)c.mx) % (unsigned)c.my),
              k = (int)(u / ((unsigned)c.mx * (unsigned)c.my));
    const long long n = gidx(c, i, j, k);
    cs[n] = dyn_clip(box ? *box : cs[n], nvert[n], max_cs);
  }
}

// (4) the 1/aj-weighted mean of lCS (ct) over the 27 nodes around interior
// nodes with nvert < 0.1 (les.c:1302-1333).
static __global__ void dyn_avg_kernel(const DevCfg c, const double *aj, const double *nvert, const double *ct,
                                      double *cs) {
  const long long total = (long long)(c.mx - 2) * (c.my - 2) * (c.mz - 2);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const unsigned u = (unsigned)t, nx = (unsigned)(c.mx - 2), ny = (unsigned)(c.my - 2);
    const int i = 1 + (int)(u % nx), j = 1 + (int)((u / nx) % ny), k = 1 + (int)(u / (nx * ny));
    const long long n = gidx(c, i, j, k);
    if (!(nvert[n] < 0.1)) continue;
    double vs = 0.0, ws = 0.0;
    for (int R = 0; R < 3; R++)
      for (int Q = 0; Q < 3; Q++)
        for (int P = 0; P < 3; P++) {
          const long long m = gidx(c, i + P - 1, j + Q - 1, k + R - 1);
          const double w = 1. / aj[m];
          vs += w * ct[m];
          ws += w;
        }
    cs[n] = vs / ws;
  }
}

// ------------------------------------------------------ launch sequence ----
// The options of the model (the -les value, -max_cs, -i/-j/-k_homo_filter
// and the test-filter width ratio of -testfilter_ik).
struct DynOpts {
  int les;
  double max_cs, tf_mult;
  int i_homo, j_homo, k_homo;
};
// The plane pointers of one block: d a device table of 14 (du/dx .. dw/dz,
// |S|, LM, MM, CS, lCS), the rest the same planes as host-held pointers.
struct DynPlanes {
  double *const *d;
  double *sabs, *lm, *mm, *cs, *ct;
};

static inline int dyn_grid(long long work, int sms) {
  long long b = (work + 255) / 256, cap = (long long)sms * 8;
  return (int)(b > cap ? cap : (b < 1 ? 1 : b));
}

// Compute_Smagorinsky_Constant_1 with a dynamic -les on one block, enqueued
// on `st`: q the current state, qu the last CalcUCat state (nullptr: zero
// velocity), met the 9 metric planes (device table).  CS ends in P.cs.  The
// kernels' dynamic shared memory (DYN_LM_SMEM) must have been opted in by the
// calling translation unit.
static cudaError_t dyn_cs_enqueue(const DevCfg &dc, const DynOpts &o, const double *const *q, const double *const *qu,
                                  const double *const *met, const double *aj, const double *nvert, const DynPlanes &P,
                                  int sms, cudaStream_t st) {
  double *const *D = P.d;
  const long long plane = dc.plane;
  const int gp = dyn_grid(plane, sms);
  const long long shell = shell_count(dc);
  const long long faces = (long long)(dc.my - 2) * (dc.mz - 2) + (long long)(dc.mx - 2) * (dc.mz - 2) +
                          (long long)(dc.mx - 2) * (dc.my - 2);
  dyn_grad_kernel<<<gp, 256, 0, st>>>(dc, q, qu, met, aj, nvert, D, P.sabs);
  ghost_fill_kernel<<<dyn_grid(shell, sms), 256, 0, st>>>(dc, D, 10);  // DMLocalToLocal
  dyn_copy_kernel<<<dyn_grid(faces, sms), 256, 0, st>>>(dc, D, 9);
  // LM / MM: zero on the whole box (the reference's VecSet), then the interior tiles
  cudaError_t e = cudaMemsetAsync(P.lm, 0, sizeof(double) * plane, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(P.mm, 0, sizeof(double) * plane, st);
  if (e != cudaSuccess) return e;
  {
    const int kc = dc.mz - 2 < 8 ? dc.mz - 2 : 8;
    const dim3 grid((dc.mx - 2 + DYN_BX - 1) / DYN_BX, (dc.my - 2 + DYN_BY - 1) / DYN_BY, (dc.mz - 2 + kc - 1) / kc);
    dyn_lm_tiled_kernel<<<grid, dim3(DYN_BX, DYN_BY), DYN_LM_SMEM, st>>>(dc, q, qu, aj, nvert, (const double *const *)D,
                                                                          P.sabs, P.lm, P.mm, kc, o.tf_mult);
  }
  ghost_fill_kernel<<<dyn_grid(shell, sms), 256, 0, st>>>(dc, D + 10, 2);
  const bool homo = o.i_homo || o.j_homo || o.k_homo;
  const bool pointwise = homo || o.les == 3;  // les.c:916-922
  const long long owned = (long long)dc.mx * dc.my * dc.mz;
  dyn_cs_kernel<<<dyn_grid(owned, sms), 256, 0, st>>>(dc, nvert, P.lm, P.mm, P.cs, o.max_cs, pointwise ? 1 : 0,
                                                      homo ? 0 : 1);
  if (homo) {
    // the reference's homogeneous branches in order; with all three filters
    // the box value overwrites every node the plane means wrote
    const bool box = o.i_homo && o.j_homo && o.k_homo;
    if (o.i_homo && o.k_homo && !box) dyn_homo_plane_kernel<<<dc.my - 2, DYN_RED, 0, st>>>(dc, nvert, P.lm, P.mm, P.cs);
    if (o.i_homo && !o.k_homo)
      dyn_homo_line_kernel<<<dyn_grid((long long)(dc.my - 2) * (dc.mz - 2), sms), 256, 0, st>>>(dc, nvert, P.lm, P.mm,
                                                                                                 P.cs);
    // lCS is scratch here: 2 * nparts + 1 doubles of its plane
    const long long np = (plane - 1) / 2 < 2LL * sms ? (plane - 1) / 2 : 2LL * sms;
    const int nparts = (int)(np < 1 ? 1 : np);
    if (box) {
      dyn_homo_box_partial_kernel<<<nparts, DYN_RED, 0, st>>>(dc, P.lm, P.mm, P.ct);
      dyn_homo_box_final_kernel<<<1, DYN_RED, 0, st>>>(P.ct, nparts);
    }
    dyn_clip_kernel<<<dyn_grid(owned, sms), 256, 0, st>>>(dc, nvert, P.cs, o.max_cs, box ? P.ct + 2 * nparts : nullptr);
  }
  if (pointwise) return cudaGetLastError();  // no final weighted mean (les.c:1302)
  e = cudaMemcpyAsync(P.ct, P.cs, sizeof(double) * plane, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return e;
  ghost_fill_kernel<<<dyn_grid(shell, sms), 256, 0, st>>>(dc, D + 13, 1);  // DMGlobalToLocal
  dyn_copy_kernel<<<dyn_grid(faces, sms), 256, 0, st>>>(dc, D + 13, 1);
  dyn_avg_kernel<<<dyn_grid((long long)(dc.mx - 2) * (dc.my - 2) * (dc.mz - 2), sms), 256, 0, st>>>(dc, aj, nvert, P.ct,
                                                                                                     P.cs);
  return cudaGetLastError();
}

}  // namespace cb
