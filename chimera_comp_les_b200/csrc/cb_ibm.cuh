// Immersed-boundary interpolation on the device (ibm_interpolation_advanced,
// ibm_iso.c:2572-2880; wall models noslip / freeslip, wallfunction.c:12-48).
//
// The host-built list (one entry per interface node: three donor nodes with
// weights, the surface element of the interception point with its vertex
// weights, the distances node -> surface and surface -> donor point) lives in
// SoA arrays.  A sweep is two launches: every entry reads its donors from the
// state as the previous sweep left it (the reference reads lQ / lP and writes
// Q / P, then scatters Q -> lQ) and writes its new conserved values into a
// compact buffer; the second launch stores them at the node and at its
// periodic ghost images.  Five sweeps (itr_tmp, ibm_iso.c:2616).
//
// Pressures live in a plane P holding the reference's P / lP: the EqOfState
// after the last stage, overwritten at interface nodes (and their ghost
// images) by each sweep's interpolated pressure, which donors read.
#pragma once
#include "cb_common.cuh"

namespace cb {

constexpr int IBM_SWEEPS = 5;
// per-entry doubles, SoA (w[a * n + e]): cr1 cr2 cr3 cs1 cs2 cs3 sb sc dx dy dz
// with sb = d_s, sc = d_s + d_i and (dx, dy, dz) = node coordinates - pmin
constexpr int IBM_NW = 11;

struct IbmDev {
  int n;
  const int4 *node;       // i, j, k of the interface node; w: surface element (-1: none)
  const long long *don;   // donor offsets into a padded plane, 3 per entry
  const double *w;        // IBM_NW x n
  const int *tri;         // nv1, nv2, nv3 of each element
  const double *nf;       // element normals, 3 per element
  const double *u, *uold; // vertex velocities of this and the previous step, 3 per vertex
  double *out;            // 6 x n: the sweep's conserved values and pressure
};

// One sweep over the list: new Q of every interface node from the state q.
// slip: freeslip (inviscid or wallfunction 3), else noslip; iso1: isothermal
// wall with Tb = 1 (rho = p gamma Ma^2), else d rho / dn = 0.
static __global__ void __launch_bounds__(256) ibm_interp_kernel(const DevCfg c, const double *const *q, const double *P,
                                                                 IbmDev b, int add_dundt, int twoD, int slip, int iso1) {
  const int n = b.n;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int cell = b.node[e].w;
    const long long d1 = b.don[3 * e], d2 = b.don[3 * e + 1], d3 = b.don[3 * e + 2];
    const double sk1 = b.w[e], sk2 = b.w[n + e], sk3 = b.w[2 * n + e];
    const double sb = b.w[6 * n + e], sc = b.w[7 * n + e];
    // direction interception point -> node (ibm_iso.c:2662-2681)
    double nfx = twoD == 1 ? 0. : b.w[8 * n + e];
    double nfy = twoD == 2 ? 0. : b.w[9 * n + e];
    double nfz = twoD == 3 ? 0. : b.w[10 * n + e];
    const double dr = sqrt(nfx * nfx + nfy * nfy + nfz * nfz);
    if (dr < 0.000000001) {
      if (cell >= 0) { nfx = b.nf[3 * cell]; nfy = b.nf[3 * cell + 1]; nfz = b.nf[3 * cell + 2]; }
      else { nfx = 0.; nfy = 0.; nfz = 0.; }
    } else {
      nfx = nfx / dr; nfy = nfy / dr; nfz = nfz / dr;
    }
    // wall velocity at the interception point, now and one step back
    double Ua[3] = {0., 0., 0.}, Ua_n = 0., Ua_nold = 0.;
    if (cell >= 0) {
      const double cs1 = b.w[3 * n + e], cs2 = b.w[4 * n + e], cs3 = b.w[5 * n + e];
      const int v1 = b.tri[3 * cell], v2 = b.tri[3 * cell + 1], v3 = b.tri[3 * cell + 2];
#pragma unroll
      for (int d = 0; d < 3; d++) Ua[d] = b.uold[3 * v1 + d] * cs1 + b.uold[3 * v2 + d] * cs2 + b.uold[3 * v3 + d] * cs3;
      Ua_nold = Ua[0] * nfx + Ua[1] * nfy + Ua[2] * nfz;
#pragma unroll
      for (int d = 0; d < 3; d++) Ua[d] = b.u[3 * v1 + d] * cs1 + b.u[3 * v2 + d] * cs2 + b.u[3 * v3 + d] * cs3;
      Ua_n = Ua[0] * nfx + Ua[1] * nfy + Ua[2] * nfz;
    }
    // donor-point velocity (ibm_iso.c:2704-2706)
    double Uc[3];
#pragma unroll
    for (int d = 0; d < 3; d++)
      Uc[d] = q[1 + d][d1] / q[0][d1] * sk1 + q[1 + d][d2] / q[0][d2] * sk2 + q[1 + d][d3] / q[0][d3] * sk3;
    double Ub[3];
    if (slip) {
      const double Uan = Ua[0] * nfx + Ua[1] * nfy + Ua[2] * nfz;
      const double Ucn = Uc[0] * nfx + Uc[1] * nfy + Uc[2] * nfz;
      const double Ubn = Uan + (Ucn - Uan) * sb / sc;
      Ub[0] = (Uc[0] - Ucn * nfx) + Ubn * nfx;
      Ub[1] = (Uc[1] - Ucn * nfy) + Ubn * nfy;
      Ub[2] = (Uc[2] - Ucn * nfz) + Ubn * nfz;
    } else {
#pragma unroll
      for (int d = 0; d < 3; d++) Ub[d] = sb / sc * (Uc[d] - Ua[d]) + Ua[d];
    }
    double pb = P[d1] * sk1 + P[d2] * sk2 + P[d3] * sk3;  // ibm_iso.c:2737-2741
    if (twoD == 1) Ub[0] = 0.;
    if (twoD == 2) Ub[1] = 0.;
    if (twoD == 3) Ub[2] = 0.;
    double rho;
    if (iso1) rho = pb * (c.gamma * c.ma * c.ma) / 1.0;  // Tb = 1 (ibm_iso.c:2795-2803)
    else rho = q[0][d1] * sk1 + q[0][d2] * sk2 + q[0][d3] * sk3;
    if (add_dundt) pb += rho * (Ua_n - Ua_nold) / c.dt * (sc - sb);
    const double ru = rho * Ub[0], rv = rho * Ub[1], rw = rho * Ub[2];
    b.out[e] = rho;
    b.out[n + e] = ru;
    b.out[2 * n + e] = rv;
    b.out[3 * n + e] = rw;
    b.out[4 * n + e] = pb / (c.gamma - 1) + 0.5 * (ru * ru + rv * rv + rw * rw) / rho;
    b.out[5 * n + e] = pb;
  }
}

// Store the sweep's values (Q and P) at each interface node and at every ghost
// image of it in the periodic directions (the DMGlobalToLocal of Q and P that
// ends a sweep).
static __global__ void __launch_bounds__(256) ibm_scatter_kernel(const DevCfg c, double *const *q, double *P, IbmDev b) {
  const int n = b.n;
  const bool per[3] = {c.bctype[0] == 7, c.bctype[2] == 7, c.bctype[4] == 7};
  const int m[3] = {c.mx, c.my, c.mz};
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int4 nd = b.node[e];
    const int x[3] = {nd.x, nd.y, nd.z};
    double v[6];
#pragma unroll
    for (int f = 0; f < 6; f++) v[f] = b.out[f * n + e];
    for (int a = -1; a <= 1; a++)
      for (int bb = -1; bb <= 1; bb++)
        for (int cc = -1; cc <= 1; cc++) {
          const int sh[3] = {a, bb, cc};
          int y[3];
          bool ok = true;
#pragma unroll
          for (int d = 0; d < 3; d++) {
            y[d] = x[d] + sh[d] * m[d];
            if (sh[d] != 0 && !per[d]) ok = false;
            if (y[d] < -2 || y[d] > m[d] + 1) ok = false;
          }
          if (!ok) continue;
          const long long g = gidx(c, y[0], y[1], y[2]);
#pragma unroll
          for (int f = 0; f < 5; f++) q[f][g] = v[f];
          P[g] = v[5];
        }
  }
}

}  // namespace cb
