// Immersed-boundary interpolation on the device (ibm_interpolation_advanced,
// ibm_iso.c:2572-2880; wall models noslip / freeslip, wallfunction.c:12-48,
// and the hydset log law of -wallfunction 2, wallfunction.c:49-100, 376-420).
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
  double *ustar;          // n: u_tau of the log-law wall (-wallfunction 2)
  // -isothermal 2 only (else null): the list keeps every entry, `last` marks
  // the entry that writes its node (a node listed twice: the later one);
  // iso holds IBM_ISO_NS x n per-entry terms and the chain's results, pa the
  // pressure the chain carries from one sweep to the next
  const unsigned char *last;
  double *iso;
  double *pa;
};

// -isothermal 2 per-entry terms (iso[a * n + e]): interpolated p, Lambda1/sc,
// rhoc a (Uc - Ua).n, Qold's rho at the node, Tb, Ub (3), Ua_n - Ua_nold;
// then the chain's rho and p
constexpr int IBM_ISO_NS = 11;

// The hydset log law (-wallfunction 2): kappa 0.41, B 5.5 (wallfunction.c:10),
// roughness ks; the reference's operation order, u_tau by Newton's method
// with a central-difference derivative, at most 30 iterations.
constexpr double WF_KAPPA = 0.41, WF_B = 5.5;
__device__ __forceinline__ double wf_E(double utau, double ks, double nu) {  // E_coeff, wallfunction.c:49-56
  const double kplus = utau * ks / nu;
  double dB;
  if (kplus <= 2.25) dB = 0.0;
  else if (kplus > 2.25 && kplus < 90.) dB = (WF_B - 8.5 + 1. / WF_KAPPA * log(kplus)) * sin(0.4258 * (log(kplus) - 0.811));
  else dB = WF_B - 8.5 + 1. / WF_KAPPA * log(kplus);
  return exp(WF_KAPPA * (WF_B - dB));
}
__device__ __forceinline__ double wf_u(double nu, double y, double utau, double ks) {  // u_hydset_roughness
  const double yplus = utau * y / nu;
  if (yplus <= 11.53) return utau * yplus;
  if (yplus <= 300) return utau / WF_KAPPA * log(wf_E(utau, ks, nu) * yplus);
  return -1.;
}
__device__ __forceinline__ double wf_f(double nu, double u, double y, double utau0, double ks) {  // f_hydset
  const double yplus = utau0 * y / nu;
  if (yplus <= 11.53) return utau0 * yplus - u;
  return utau0 * (1. / WF_KAPPA * log(wf_E(utau0, ks, nu) * yplus)) - u;
}
static __device__ __noinline__ double wf_find_utau(double nu, double u, double y, double guess, double ks) {
  const double eps = 1.e-7;  // find_utau_hydset, wallfunction.c:85-100
  double utau = guess, utau0 = guess;
  for (int ii = 0; ii < 30; ii++) {
    const double df = (wf_f(nu, u, y, utau0 + eps, ks) - wf_f(nu, u, y, utau0 - eps, ks)) / (2. * eps);
    utau = utau0 - wf_f(nu, u, y, utau0, ks) / df;
    if (fabs(utau - utau0) < 1.e-7) break;
    utau0 = utau;
  }
  return utau;
}

// One sweep over the list: new Q of every interface node from the state q.
// slip: freeslip (inviscid or wallfunction 3), else noslip; iso1: isothermal
// wall with Tb = 1 (rho = p gamma Ma^2), else d rho / dn = 0.
// wf2: the log-law wall of -wallfunction 2, which takes precedence over slip
// (ibm_iso.c:2708-2728).
// iso2: -isothermal 2, whose density and pressure come from the chain
// (ibm_iso2_chain_kernel) over the terms this kernel stores; rho_old: the
// density of Qold (-isothermal 2 only); a_sound: sqrt(Twall / Ma^2).
static __global__ void __launch_bounds__(256) ibm_interp_kernel(const DevCfg c, const double *const *q, const double *P,
                                                                 IbmDev b, int add_dundt, int twoD, int slip, int iso1,
                                                                 int wf2, const double *rho_old, double a_sound) {
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
    if (wf2) {  // wall_function_loglaw(user, 1.e-16, ...), wallfunction.c:376-420
      const double sbc = sb / sc;
      const double u_c = Uc[0] - Ua[0], v_c = Uc[1] - Ua[1], w_c = Uc[2] - Ua[2];
      const double un = u_c * nfx + v_c * nfy + w_c * nfz;
      double ut = u_c - un * nfx, vt = v_c - un * nfy, wt = w_c - un * nfz;
      const double ut_mag = sqrt(ut * ut + vt * vt + wt * wt);
      const double us = wf_find_utau(c.inv_ren, ut_mag, sc, 0.001, 1.e-16);
      double model = wf_u(c.inv_ren, sb, us, 1.e-16);
      if (model < 0.) model = ut_mag;
      if (ut_mag > 1.e-10) {
        ut *= model / ut_mag;
        vt *= model / ut_mag;
        wt *= model / ut_mag;
      } else {
        ut = vt = wt = 0;
      }
      Ub[0] = ut + (sbc * un) * nfx + Ua[0];
      Ub[1] = vt + (sbc * un) * nfy + Ua[1];
      Ub[2] = wt + (sbc * un) * nfz + Ua[2];
      b.ustar[e] = us;
    } else if (slip) {
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
    if (rho_old) {  // -isothermal 2 (ibm_iso.c:2744-2786): terms that do not depend on Pa
      const double gm2 = c.gamma * c.ma * c.ma;
      const double rhoc = q[0][d1] * sk1 + q[0][d2] * sk2 + q[0][d3] * sk3;
      double Tc = pb / rhoc * gm2;
      if (Tc < 0.) Tc = 0.;
      const int4 nd = b.node[e];
      double *S = b.iso;
      S[e] = pb;
      S[n + e] = (Ua_n - a_sound) / sc;
      S[2 * n + e] = rhoc * a_sound * ((Uc[0] - Ua[0]) * nfx + (Uc[1] - Ua[1]) * nfy + (Uc[2] - Ua[2]) * nfz);
      S[3 * n + e] = rho_old[gidx(c, nd.x, nd.y, nd.z)];
      S[4 * n + e] = (Tc - c.twall) * sb / sc + c.twall;
      S[5 * n + e] = Ub[0];
      S[6 * n + e] = Ub[1];
      S[7 * n + e] = Ub[2];
      S[8 * n + e] = Ua_n - Ua_nold;
      continue;
    }
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

// -isothermal 2: the entries in list order, each reading the pressure Pa the
// previous entry left (its own at the first sweep; across sweeps the last
// entry's), as the reference's single variable Pa does:
//   L1 = Lambda1/sc ((p - Pa) - rhoc a (Uc - Ua).n),
//   rho = rho_old - dt L1 / a / a,  p = rho Tb / (gamma Ma^2),  Pa = p.
// One block: each chunk of entries is staged in shared memory by all threads,
// thread 0 walks it, all threads store the results.  The loop is bounded by
// the list length.
constexpr int IBM_CHAIN_NT = 256;
static __global__ void __launch_bounds__(IBM_CHAIN_NT) ibm_iso2_chain_kernel(const DevCfg c, IbmDev b, int first,
                                                                            double a_sound) {
  __shared__ double sp[IBM_CHAIN_NT], sc1[IBM_CHAIN_NT], sx[IBM_CHAIN_NT], sr[IBM_CHAIN_NT], st[IBM_CHAIN_NT];
  const int n = b.n;
  const double *S = b.iso;
  double *R = b.iso + 9 * (size_t)n, *PF = b.iso + 10 * (size_t)n;
  const double gm2 = c.gamma * c.ma * c.ma;
  double Pa = first ? 0. : *b.pa;  // thread 0's copy is the one that counts
  for (int e0 = 0; e0 < n; e0 += IBM_CHAIN_NT) {
    const int e = e0 + threadIdx.x;
    if (e < n) {
      sp[threadIdx.x] = S[e];
      sc1[threadIdx.x] = S[n + e];
      sx[threadIdx.x] = S[2 * n + e];
      sr[threadIdx.x] = S[3 * n + e];
      st[threadIdx.x] = S[4 * n + e];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int m = min(IBM_CHAIN_NT, n - e0);
      for (int t = 0; t < m; t++) {
        const double p = sp[t];
        if (first) Pa = p;
        const double L1 = sc1[t] * ((p - Pa) - sx[t]);
        const double rho = sr[t] - c.dt * L1 / a_sound / a_sound;
        const double pf = rho * st[t] / gm2;
        Pa = pf;
        sr[t] = rho;
        st[t] = pf;
      }
    }
    __syncthreads();
    if (e < n) {
      R[e] = sr[threadIdx.x];
      PF[e] = st[threadIdx.x];
    }
    __syncthreads();  // the next chunk overwrites the staging
  }
  if (threadIdx.x == 0) *b.pa = Pa;
}

// -isothermal 2: each entry's conserved values from the chain's rho and p.
static __global__ void __launch_bounds__(256) ibm_iso2_finish_kernel(const DevCfg c, IbmDev b, int add_dundt) {
  const int n = b.n;
  const double *S = b.iso;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const double sb = b.w[6 * n + e], sc = b.w[7 * n + e];
    const double rho = S[9 * (size_t)n + e];
    double pb = S[10 * (size_t)n + e];
    if (add_dundt) pb += rho * S[8 * n + e] / c.dt * (sc - sb);
    const double ru = rho * S[5 * n + e], rv = rho * S[6 * n + e], rw = rho * S[7 * n + e];
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
    if (b.last && !b.last[e]) continue;  // a node listed twice: its later entry writes it
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
