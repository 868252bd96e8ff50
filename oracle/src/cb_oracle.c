/*
 * CPU restatement of the reference's compressible RHS + SSP-RK stage update
 * (TEST INFRASTRUCTURE ONLY -- the checker, never the product).
 *
 * Each routine cites the reference lines it restates.  The reference writes
 * each sweep three times (xi, eta, zeta); here one direction-generic routine
 * serves all three and the per-direction differences of the reference are
 * reproduced explicitly (marked "quirk").  Arithmetic follows the reference's
 * expression order so results agree to rounding.
 */
#include "cb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define BLANKWALL 2.9 /* rhs.c:2598, 3261 */
#define BLANK 0.1     /* rhs.c:2598 */
#define SOLID 0.5     /* rhs.c:1407 */
#define INNERBLANK 7. /* rhs.c:1408 */
#define GAMMA_CONV 1.4 /* formConvection/LES hard-code gamma=1.4 (rhs.c:2596, 3257) */

typedef struct {
  int m[3];          /* mx, my, mz */
  int g[3];          /* padded extents m+4 */
  ptrdiff_t s[3];    /* strides */
  size_t n;          /* padded node count */
  int per[3];        /* periodic flags */
} geom;

static geom mkgeom(const cbo_config *c) {
  geom G;
  G.m[0] = c->mx; G.m[1] = c->my; G.m[2] = c->mz;
  for (int d = 0; d < 3; d++) G.g[d] = G.m[d] + 4;
  G.s[0] = 1; G.s[1] = G.g[0]; G.s[2] = (ptrdiff_t)G.g[0] * G.g[1];
  G.n = (size_t)G.g[0] * G.g[1] * G.g[2];
  /* init.c:148-199: a direction is periodic iff its low-side bctype is 7 */
  G.per[0] = c->bctype[0] == 7; G.per[1] = c->bctype[2] == 7; G.per[2] = c->bctype[4] == 7;
  return G;
}

static inline ptrdiff_t IX(const geom *G, int i, int j, int k) {
  return ((ptrdiff_t)(k + 2) * G->g[1] + (j + 2)) * G->g[0] + (i + 2);
}

/* solvers.c:247: the stage loop runs istage < fluxorder (1: Euler, 2: RK2, 3: RK3) */
int cbo_nstages(const cbo_config *c) { return c->fluxorder; }

/* ------------------------------------------------------------------------ */
/* DMGlobalToLocal wrap-around for periodic directions                        */
/* ------------------------------------------------------------------------ */
void cbo_fill_ghosts(const cbo_config *c, double *f) {
  geom G = mkgeom(c);
  for (int k = -2; k < G.m[2] + 2; k++)
    for (int j = -2; j < G.m[1] + 2; j++)
      for (int i = -2; i < G.m[0] + 2; i++) {
        int x[3] = {i, j, k}, w[3];
        int skip = 0, moved = 0;
        for (int d = 0; d < 3; d++) {
          w[d] = x[d];
          if (x[d] < 0 || x[d] >= G.m[d]) {
            if (!G.per[d]) { skip = 1; break; }
            w[d] = ((x[d] % G.m[d]) + G.m[d]) % G.m[d];
            moved = 1;
          }
        }
        if (skip || !moved) continue;
        f[IX(&G, i, j, k)] = f[IX(&G, w[0], w[1], w[2])];
      }
}

/* ------------------------------------------------------------------------ */
/* FormMetrics  (metrics.c:3-246)                                            */
/* ------------------------------------------------------------------------ */
void cbo_metrics(const cbo_config *c, const double *const X[3], double *const csi[3],
                 double *const eta[3], double *const zet[3], double *aj) {
  geom G = mkgeom(c);
  const int mx = G.m[0], my = G.m[1], mz = G.m[2];
  for (int d = 0; d < 3; d++) {
    memset(csi[d], 0, G.n * sizeof(double));
    memset(eta[d], 0, G.n * sizeof(double));
    memset(zet[d], 0, G.n * sizeof(double));
  }
  memset(aj, 0, G.n * sizeof(double));
  const ptrdiff_t si = G.s[0], sj = G.s[1], sk = G.s[2];
#define DC(a, n) (0.5 * (X[a][(n) + si] - X[a][(n) - si]))
#define DE(a, n) (0.5 * (X[a][(n) + sj] - X[a][(n) - sj]))
#define DZ(a, n) (0.5 * (X[a][(n) + sk] - X[a][(n) - sk]))
  /* metrics.c:52-70: csi = de x dz on k,j interior, all i */
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 0; i < mx; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        double dxde = DE(0, n), dyde = DE(1, n), dzde = DE(2, n);
        double dxdz = DZ(0, n), dydz = DZ(1, n), dzdz = DZ(2, n);
        csi[0][n] = dyde * dzdz - dzde * dydz;
        csi[1][n] = -dxde * dzdz + dzde * dxdz;
        csi[2][n] = dxde * dydz - dyde * dxdz;
      }
  /* metrics.c:73-92: eta = dz x dc on k,i interior, all j */
  for (int k = 1; k < mz - 1; k++)
    for (int j = 0; j < my; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        double dxdc = DC(0, n), dydc = DC(1, n), dzdc = DC(2, n);
        double dxdz = DZ(0, n), dydz = DZ(1, n), dzdz = DZ(2, n);
        eta[0][n] = dydz * dzdc - dzdz * dydc;
        eta[1][n] = -dxdz * dzdc + dzdz * dxdc;
        eta[2][n] = dxdz * dydc - dydz * dxdc;
      }
  /* metrics.c:95-113: zet = dc x de on j,i interior, all k */
  for (int k = 0; k < mz; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        double dxdc = DC(0, n), dydc = DC(1, n), dzdc = DC(2, n);
        double dxde = DE(0, n), dyde = DE(1, n), dzde = DE(2, n);
        zet[0][n] = dydc * dzde - dzdc * dyde;
        zet[1][n] = -dxdc * dzde + dzdc * dxde;
        zet[2][n] = dxdc * dyde - dydc * dxde;
      }
  /* metrics.c:116-136: aj = 1/det on the interior */
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        double dxdc = DC(0, n), dydc = DC(1, n), dzdc = DC(2, n);
        double dxde = DE(0, n), dyde = DE(1, n), dzde = DE(2, n);
        double dxdz = DZ(0, n), dydz = DZ(1, n), dzdz = DZ(2, n);
        double det = dxdc * (dyde * dzdz - dzde * dydz) - dydc * (dxde * dzdz - dzde * dxdz) +
                     dzdc * (dxde * dydz - dyde * dxdz);
        aj[n] = 1. / det;
      }
#undef DC
#undef DE
#undef DZ
  /* metrics.c:138-246: boundary layers copied from the inward neighbour, in
   * the order i-low, i-high, j-low, j-high, k-low, k-high (later wins). */
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++) {
      ptrdiff_t n = IX(&G, 0, j, k);
      for (int a = 0; a < 3; a++) { eta[a][n] = eta[a][n + si]; zet[a][n] = zet[a][n + si]; }
      aj[n] = aj[n + si];
    }
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++) {
      ptrdiff_t n = IX(&G, mx - 1, j, k);
      for (int a = 0; a < 3; a++) { eta[a][n] = eta[a][n - si]; zet[a][n] = zet[a][n - si]; }
      aj[n] = aj[n - si];
    }
  for (int k = 0; k < mz; k++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, 0, k);
      for (int a = 0; a < 3; a++) { csi[a][n] = csi[a][n + sj]; zet[a][n] = zet[a][n + sj]; }
      aj[n] = aj[n + sj];
    }
  for (int k = 0; k < mz; k++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, my - 1, k);
      for (int a = 0; a < 3; a++) { csi[a][n] = csi[a][n - sj]; zet[a][n] = zet[a][n - sj]; }
      aj[n] = aj[n - sj];
    }
  for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, j, 0);
      for (int a = 0; a < 3; a++) { eta[a][n] = eta[a][n + sk]; csi[a][n] = csi[a][n + sk]; }
      aj[n] = aj[n + sk];
    }
  for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, j, mz - 1);
      for (int a = 0; a < 3; a++) { eta[a][n] = eta[a][n - sk]; csi[a][n] = csi[a][n - sk]; }
      aj[n] = aj[n - sk];
    }
  /* metrics.c:264-271: scatter to the ghosted local vectors */
  for (int a = 0; a < 3; a++) {
    cbo_fill_ghosts(c, csi[a]);
    cbo_fill_ghosts(c, eta[a]);
    cbo_fill_ghosts(c, zet[a]);
  }
  cbo_fill_ghosts(c, aj);
}

/* ------------------------------------------------------------------------ */
/* EqOfState  (rhs.c:4820-4870)                                              */
/* ------------------------------------------------------------------------ */
static inline double eos(double g, double r, double ru, double rv, double rw, double re) {
  return (g - 1) * (re - 0.5 * (ru * ru + rv * rv + rw * rw) / r);
}

void cbo_eos(const cbo_config *c, const double *const q[5], double *p) {
  geom G = mkgeom(c);
  for (size_t n = 0; n < G.n; n++)
    p[n] = q[0][n] != 0.0 ? eos(c->gamma, q[0][n], q[1][n], q[2][n], q[3][n], q[4][n]) : 0.0;
}

/* ------------------------------------------------------------------------ */
/* Hybrid weights  (rhs.c:3322-3441, sensor off)                             */
/* ------------------------------------------------------------------------ */
void cbo_sigma(const cbo_config *c, double *const sig[3]) {
  geom G = mkgeom(c);
  for (size_t n = 0; n < G.n; n++) { sig[0][n] = c->s_x; sig[1][n] = c->s_y; sig[2][n] = c->s_z; }
  /* rhs.c:3415-3432: interior nodes get y = z = min(z, y); the curvature
   * tests there never fire on a uniform field. */
  double mzy = c->s_z < c->s_y ? c->s_z : c->s_y;
  for (int k = 1; k < G.m[2] - 1; k++)
    for (int j = 1; j < G.m[1] - 1; j++)
      for (int i = 1; i < G.m[0] - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        sig[2][n] = mzy;
        sig[1][n] = mzy;
      }
  for (int a = 0; a < 3; a++) cbo_fill_ghosts(c, sig[a]);
}

/* compute_ri / sigma_cent (rhs.c:2334-2358): smoothness ratio of two
 * neighbouring differences and the tanh ramp from it. */
static double compute_ri(double fR, double f0, double fL, double ks) {
  double dfL = fL - f0, dfR = f0 - fR;
  return (fabs(2 * dfL * dfR) + ks) / (dfL * dfL + dfR * dfR + ks);
}
static double sigma_cent(double fL, double f0, double fR, double fRR, double ks) {
  double rL = compute_ri(fL, f0, fR, ks), rR = compute_ri(f0, fR, fRR, ks);
  double r = (rR < rL) ? rR : rL;       /* PetscMin(rR, rL) */
  double rd = 0.5;
  double rmax = (rd < r) ? r : rd;      /* PetscMax(rd, r) */
  return 0.5 + 0.5 * tanh(3.0 * (r - rd) / rmax) / tanh(3.0);
}
#define PMIN(a, b) (((a) < (b)) ? (a) : (b))
#define PMAX(a, b) (((a) < (b)) ? (b) : (a))

/* Hybrid weights with the sensor on (rhs.c:3328-3433): per interior node the
 * ramp of the pressure smoothness along each direction (x for 2 < i < mx-4,
 * y for 4 < j < my-4, z everywhere in a periodic k), clipped to
 * [s_min, s]; a product filter of square roots of neighbour pairs; then the
 * curvature rule and y = z = min(y, z).  Boundary nodes keep (s_x, s_y, s_z).
 * p: the ghosted pressure formConvectionLES reads as lP. */
void cbo_sigma_sensor_p(const cbo_config *c, const double *p, double *const sig[3]) {
  geom G = mkgeom(c);
  double *ls[3];
  for (int a = 0; a < 3; a++) ls[a] = (double *)malloc(G.n * sizeof(double));
  const double ks = c->sigma_thrsh;
  const ptrdiff_t si = 1, sj = G.m[0] + 4, sk = (ptrdiff_t)(G.m[0] + 4) * (G.m[1] + 4);
  const int mx = G.m[0], my = G.m[1], mz = G.m[2];
  for (size_t n = 0; n < G.n; n++) { sig[0][n] = c->s_x; sig[1][n] = c->s_y; sig[2][n] = c->s_z; }
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        if (c->abc != 0 && k > c->abc) sig[0][n] = 0.; /* -ABC absorbing layer (rhs.c:3341) */
        else if (i < mx - 4 && i > 2) sig[0][n] = sigma_cent(p[n - si], p[n], p[n + si], p[n + 2 * si], ks);
        sig[0][n] = PMIN(c->s_x, sig[0][n]);
        sig[0][n] = PMAX(c->s_x_min, sig[0][n]);
      }
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        if (c->abc != 0 && k > c->abc) sig[2][n] = 0.; /* rhs.c:3355 */
        else if (c->bctype[4] == 7 || (k < mz - 4 && k > 4))
          sig[2][n] = sigma_cent(p[n - sk], p[n], p[n + sk], p[n + 2 * sk], ks);
        sig[2][n] = PMIN(c->s_z, sig[2][n]);
        sig[2][n] = PMAX(c->s_z_min, sig[2][n]);
      }
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        if (c->abc != 0 && k > c->abc) sig[1][n] = 0.; /* rhs.c:3368 */
        else if (j < my - 4 && j > 4) sig[1][n] = sigma_cent(p[n - sj], p[n], p[n + sj], p[n + 2 * sj], ks);
        sig[1][n] = PMIN(c->s_y, sig[1][n]);
        sig[1][n] = PMAX(c->s_y_min, sig[1][n]);
      }
  /* filter with the ghosted copy (rhs.c:3382-3407) */
  for (int a = 0; a < 3; a++) {
    memcpy(ls[a], sig[a], G.n * sizeof(double));
    cbo_fill_ghosts(c, ls[a]);
  }
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        for (int a = 0; a < 3; a++)
          sig[a][n] *= sqrt(ls[a][n - sj] * ls[a][n]) * sqrt(ls[a][n - sk] * ls[a][n + sk]) *
                       sqrt(ls[a][n - si] * ls[a][n + si]);
      }
  /* curvature rule and y = z = min (rhs.c:3415-3433) */
  for (int a = 0; a < 3; a++) {
    memcpy(ls[a], sig[a], G.n * sizeof(double));
    cbo_fill_ghosts(c, ls[a]);
  }
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        if (j < my - 4 && j > 4 && ls[1][n - sj] + ls[1][n + sj] - 2. * ls[1][n] < 0.0)
          sig[1][n] = (ls[1][n - sj] * ls[1][n] * ls[1][n]);
        if (k < mz - 4 && k > 4 && ls[2][n - sk] + ls[2][n + sk] - 2. * ls[2][n] < 0.0)
          sig[2][n] = (ls[2][n - sk] * ls[2][n + sk] * ls[2][n]);
        sig[2][n] = PMIN(sig[2][n], sig[1][n]);
        sig[1][n] = sig[2][n];
      }
  for (int a = 0; a < 3; a++) cbo_fill_ghosts(c, sig[a]);
  for (int a = 0; a < 3; a++) free(ls[a]);
}

/* The sensor on the EqOfState of q (the lP of a step without a carried
 * pressure). */
void cbo_sigma_sensor(const cbo_config *c, const double *const q[5], double *const sig[3]) {
  geom G = mkgeom(c);
  double *p = (double *)malloc(G.n * sizeof(double));
  cbo_eos(c, q, p);
  cbo_sigma_sensor_p(c, p, sig);
  free(p);
}

/* ------------------------------------------------------------------------ */
/* Reconstructions  (rhs.c:2256-2307, 2359-2461, 2498-2568)                  */
/* ------------------------------------------------------------------------ */
static inline double sgn(double a) { return (a >= 0) ? ((a == 0) ? 0 : 1) : -1; }
static inline double minmod(double a, double b) {
  if (a * b < 0) return 0.;
  double fa = fabs(a), fb = fabs(b);
  return sgn(a) * ((fa < fb) ? fa : fb);
}
static inline double muscl_l(double qm, double q0, double qp) { return q0 + 0.5 * minmod(qp - q0, q0 - qm); }
static inline double muscl_r(double qm, double q0, double qp) { return q0 - 0.5 * minmod(qp - q0, q0 - qm); }

static inline double weno3_l(double qm, double q0, double qp) {
  const double d0 = 0.6666667, d1 = 0.3333333, eps = 1e-6; /* truncated weights, rhs.c:2386 */
  double r0 = 0.5 * q0 + 0.5 * qp, r1 = -0.5 * qm + 1.5 * q0;
  double b0 = (qp - q0) * (qp - q0), b1 = (qm - q0) * (qm - q0);
  double a0 = d0 / ((eps + b0) * (eps + b0)), a1 = d1 / ((eps + b1) * (eps + b1));
  double as = a0 + a1;
  return (a0 / as) * r0 + (a1 / as) * r1;
}
static inline double weno3_r(double qm, double q0, double qp) {
  const double d0 = 0.6666667, d1 = 0.3333333, eps = 1e-6;
  double r0 = 1.5 * q0 - 0.5 * qp, r1 = 0.5 * qm + 0.5 * q0;
  double b0 = (qp - q0) * (qp - q0), b1 = (qm - q0) * (qm - q0);
  double a0 = d0 / ((eps + b0) * (eps + b0)), a1 = d1 / ((eps + b1) * (eps + b1));
  double as = a0 + a1;
  return (a0 / as) * r0 + (a1 / as) * r1;
}
/* WENO5-JS (G.-S. Jiang and C.-W. Shu, "Efficient implementation of weighted
 * ENO schemes", J. Comput. Phys. 126 (1996) 202-228, eqs. 2.10-2.17 with
 * p = 2): no counterpart in the reference, whose WENO is the 3rd-order one
 * above.  Value at x_{i+1/2} from a..e = v_{i-2..i+2}:
 *   candidates (times 6)  q0 = 2a - 7b + 11c,  q1 = -b + 5c + 2d,  q2 = 2c + 5d - e
 *   smoothness            beta_k = 13/12 (second difference)^2 + 1/4 (first-derivative estimate)^2
 *   weights               alpha_k = d_k / (eps + beta_k)^2,  d = (1/10, 6/10, 3/10),  eps = 1e-6
 *   value                 (alpha0 q0 + alpha1 q1 + alpha2 q2) / (6 (alpha0 + alpha1 + alpha2))
 * The operation order here is the one the device code follows. */
double cbo_weno5(double a, double b, double c, double d, double e) {
  const double eps = 1e-6, c13 = 13.0 / 12.0;
  const double q0 = (2.0 * a - 7.0 * b) + 11.0 * c;
  const double q1 = (5.0 * c - b) + 2.0 * d;
  const double q2 = (2.0 * c + 5.0 * d) - e;
  const double t0 = (a - 2.0 * b) + c, u0 = (a - 4.0 * b) + 3.0 * c;
  const double t1 = (b - 2.0 * c) + d, u1 = b - d;
  const double t2 = (c - 2.0 * d) + e, u2 = (3.0 * c - 4.0 * d) + e;
  const double b0 = c13 * (t0 * t0) + 0.25 * (u0 * u0);
  const double b1 = c13 * (t1 * t1) + 0.25 * (u1 * u1);
  const double b2 = c13 * (t2 * t2) + 0.25 * (u2 * u2);
  const double a0 = 0.1 / ((eps + b0) * (eps + b0));
  const double a1 = 0.6 / ((eps + b1) * (eps + b1));
  const double a2 = 0.3 / ((eps + b2) * (eps + b2));
  return ((a0 * q0 + a1 * q1) + a2 * q2) / (6.0 * ((a0 + a1) + a2));
}

static inline double eno_r(double qm, double q0, double qp, int k) {
  if (k == 2) return 0.5 * q0 + 0.5 * qp;
  return -qm * 0.1666666666666666 + q0 * 0.8333333333333333 + qp * 0.3333333333333333;
}
static inline double eno_l(double qm, double q0, double qp, int k) {
  if (k == 2) return 0.5 * q0 + 0.5 * qm;
  return qm * 0.3333333333333333 + q0 * 0.8333333333333333 - qp * 0.1666666666666666;
}

/* Rusanov (local Lax-Friedrichs) flux, rhs.c:2769-2810 / 3676-3695.
 * wall_lo/wall_hi reproduce the non-LES wall tweaks (rhs.c:2779-2790). */
static void rusanov(const double QL[5], const double QR[5], double pL, double pR, const double h[3],
                    int use_qr_for_l, int ucon_r_from_l, double F[5]) {
  double uconL, uconR;
  if (use_qr_for_l)
    uconL = (h[0] * (QR[1] / QR[0]) + h[1] * (QR[2] / QR[0]) + h[2] * (QR[3] / QR[0]));
  else
    uconL = (h[0] * (QL[1] / QL[0]) + h[1] * (QL[2] / QL[0]) + h[2] * (QL[3] / QL[0]));
  if (ucon_r_from_l)
    uconR = uconL;
  else
    uconR = (h[0] * (QR[1] / QR[0]) + h[1] * (QR[2] / QR[0]) + h[2] * (QR[3] / QR[0]));
  double gii = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
  double cL = GAMMA_CONV * pL / QL[0], cR = GAMMA_CONV * pR / QR[0];
  double saL = fabs(uconL) + sqrt(fabs(cL) * gii);
  double saR = fabs(uconR) + sqrt(fabs(cR) * gii);
  double SA = (saL < saR) ? saR : saL;
  F[0] = 0.5 * (QL[0] * uconL + QR[0] * uconR) - 0.5 * SA * (QR[0] - QL[0]);
  for (int a = 0; a < 3; a++)
    F[1 + a] = 0.5 * ((QL[1 + a] * uconL + QR[1 + a] * uconR) + (pL * h[a] + pR * h[a])) -
               0.5 * SA * (QR[1 + a] - QL[1 + a]);
  F[4] = 0.5 * ((pL + QL[4]) * uconL + (pR + QR[4]) * uconR) - 0.5 * SA * (QR[4] - QL[4]);
}

/* Roe's approximate Riemann solver (P. L. Roe, J. Comput. Phys. 43, 1981)
 * on a curvilinear face with area vector h: the central part is the same
 * average of the two physical fluxes as the Rusanov flux above; the
 * dissipation is |A~|(QR - QL) of the Roe-averaged Jacobian along n = h/|h|,
 * scaled by |h|, with Harten's entropy fix on the acoustic waves
 * (A. Harten, J. Comput. Phys. 49, 1983): |l| < delta -> (l^2 + delta^2) /
 * (2 delta), delta = 0.1 c~.  gamma is the flux code's 1.4.  No counterpart
 * in the reference. */
static void roe(const double QL[5], const double QR[5], double pL, double pR, const double h[3],
                int use_qr_for_l, int ucon_r_from_l, double F[5]) {
  double uconL, uconR;
  if (use_qr_for_l)
    uconL = (h[0] * (QR[1] / QR[0]) + h[1] * (QR[2] / QR[0]) + h[2] * (QR[3] / QR[0]));
  else
    uconL = (h[0] * (QL[1] / QL[0]) + h[1] * (QL[2] / QL[0]) + h[2] * (QL[3] / QL[0]));
  if (ucon_r_from_l)
    uconR = uconL;
  else
    uconR = (h[0] * (QR[1] / QR[0]) + h[1] * (QR[2] / QR[0]) + h[2] * (QR[3] / QR[0]));
  const double g = GAMMA_CONV;
  const double area = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
  const double nx = h[0] / area, ny = h[1] / area, nz = h[2] / area;
  const double sl = sqrt(QL[0]), sr = sqrt(QR[0]), wl = sl / (sl + sr), wr = sr / (sl + sr);
  const double uL = QL[1] / QL[0], vL = QL[2] / QL[0], zL = QL[3] / QL[0];
  const double uR = QR[1] / QR[0], vR = QR[2] / QR[0], zR = QR[3] / QR[0];
  const double HL = (QL[4] + pL) / QL[0], HR = (QR[4] + pR) / QR[0];
  const double rt = sl * sr, ut = wl * uL + wr * uR, vt = wl * vL + wr * vR, zt = wl * zL + wr * zR;
  const double Ht = wl * HL + wr * HR, q2 = ut * ut + vt * vt + zt * zt;
  const double c2 = (g - 1.0) * (Ht - 0.5 * q2), ct = sqrt(fabs(c2));
  const double Unt = ut * nx + vt * ny + zt * nz;
  const double dp = pR - pL, dr = QR[0] - QL[0];
  const double du = uR - uL, dv = vR - vL, dz = zR - zL, dUn = du * nx + dv * ny + dz * nz;
  const double a1 = (dp - rt * ct * dUn) / (2.0 * c2), a2 = dr - dp / c2, a3 = (dp + rt * ct * dUn) / (2.0 * c2);
  double l1 = fabs(Unt - ct), l2 = fabs(Unt), l3 = fabs(Unt + ct);
  const double delta = 0.1 * ct;
  if (l1 < delta) l1 = (l1 * l1 + delta * delta) / (2.0 * delta);
  if (l3 < delta) l3 = (l3 * l3 + delta * delta) / (2.0 * delta);
  const double s1 = l1 * a1, s2 = l2 * a2, s3 = l3 * a3, ss = l2 * rt;
  double D[5];
  D[0] = s1 + s2 + s3;
  D[1] = s1 * (ut - ct * nx) + s2 * ut + s3 * (ut + ct * nx) + ss * (du - dUn * nx);
  D[2] = s1 * (vt - ct * ny) + s2 * vt + s3 * (vt + ct * ny) + ss * (dv - dUn * ny);
  D[3] = s1 * (zt - ct * nz) + s2 * zt + s3 * (zt + ct * nz) + ss * (dz - dUn * nz);
  D[4] = s1 * (Ht - Unt * ct) + s2 * 0.5 * q2 + s3 * (Ht + Unt * ct) + ss * (ut * du + vt * dv + zt * dz - Unt * dUn);
  F[0] = 0.5 * (QL[0] * uconL + QR[0] * uconR) - 0.5 * area * D[0];
  for (int a = 0; a < 3; a++)
    F[1 + a] = 0.5 * ((QL[1 + a] * uconL + QR[1 + a] * uconR) + (pL * h[a] + pR * h[a])) - 0.5 * area * D[1 + a];
  F[4] = 0.5 * ((pL + QL[4]) * uconL + (pR + QR[4]) * uconR) - 0.5 * area * D[4];
}

typedef struct {
  const cbo_config *c;
  geom G;
  const double *const *q;
  const double *p;
  const double *nv;
  const double *const *met[3]; /* csi, eta, zet */
} ctx_t;

static inline void ld5(const ctx_t *C, ptrdiff_t n, double o[5]) {
  for (int a = 0; a < 5; a++) o[a] = C->q[a][n];
}

/* Upwind reconstruction shared by formConvection and formConvectionLES.
 * les selects the LES variant's ENO conditions; iso_j1 applies the eta
 * isothermal j==1 substitution (rhs.c:2926-2930). */
static void recon_weno(const ctx_t *C, int d, int pos, ptrdiff_t n0, int eno_l_cond, int eno_r_cond,
                       int iso_j1, double QL[5], double QR[5], double *pL, double *pR) {
  const ptrdiff_t s = C->G.s[d];
  const int ord = C->c->eno_order;
  const double *const *q = C->q;
  const double *p = C->p;
  (void)pos;
  if (eno_l_cond) {
    for (int a = 0; a < 5; a++) QL[a] = eno_l(q[a][n0], q[a][n0 + s], q[a][n0 + 2 * s], ord);
    *pL = eno_l(p[n0], p[n0 + s], p[n0 + 2 * s], ord);
  } else {
    for (int a = 0; a < 5; a++) QL[a] = weno3_l(q[a][n0 - s], q[a][n0], q[a][n0 + s]);
    *pL = weno3_l(p[n0 - s], p[n0], p[n0 + s]);
    if (iso_j1) {
      QL[0] = eno_l(q[0][n0], q[0][n0 + s], q[0][n0 + 2 * s], ord);
      QL[4] = eno_l(q[4][n0], q[4][n0 + s], q[4][n0 + 2 * s], ord);
      *pL = eno_l(p[n0], p[n0 + s], p[n0 + 2 * s], ord);
    }
  }
  if (eno_r_cond) {
    for (int a = 0; a < 5; a++) QR[a] = eno_r(q[a][n0 - s], q[a][n0], q[a][n0 + s], ord);
    *pR = eno_r(p[n0 - s], p[n0], p[n0 + s], ord);
  } else {
    for (int a = 0; a < 5; a++) QR[a] = weno3_r(q[a][n0], q[a][n0 + s], q[a][n0 + 2 * s]);
    *pR = weno3_r(p[n0], p[n0 + s], p[n0 + 2 * s]);
  }
}

/* WENO5-JS on the face pos+1/2 (between n0 and n0+e_d) where its six-node
 * stencil pos-2 .. pos+3 lies on the DMDA's nodes 0 .. m-1 (so no stencil
 * reaches the wrap-around ghosts of a periodic direction) and holds no wall
 * node (nvert > 2.9); returns 0 when that does not hold, and the caller then
 * takes the reference's WENO3 path. */
static int recon_weno5(const ctx_t *C, int d, int pos, ptrdiff_t n0, double QL[5], double QR[5], double *pL,
                       double *pR) {
  const ptrdiff_t s = C->G.s[d];
  const int m = C->G.m[d];
  const double *nv = C->nv;
  if (pos < 2 || pos > m - 4) return 0;
  if (nv[n0 - 2 * s] > BLANKWALL || nv[n0 - s] > BLANKWALL || nv[n0 + 2 * s] > BLANKWALL ||
      nv[n0 + 3 * s] > BLANKWALL)
    return 0;
  const double *const *q = C->q;
  const double *p = C->p;
  for (int a = 0; a < 5; a++) {
    const double *v = q[a];
    QL[a] = cbo_weno5(v[n0 - 2 * s], v[n0 - s], v[n0], v[n0 + s], v[n0 + 2 * s]);
    QR[a] = cbo_weno5(v[n0 + 3 * s], v[n0 + 2 * s], v[n0 + s], v[n0], v[n0 - s]);
  }
  *pL = cbo_weno5(p[n0 - 2 * s], p[n0 - s], p[n0], p[n0 + s], p[n0 + 2 * s]);
  *pR = cbo_weno5(p[n0 + 3 * s], p[n0 + 2 * s], p[n0 + s], p[n0], p[n0 - s]);
  return 1;
}

static void recon_muscl(const ctx_t *C, int d, ptrdiff_t n0, double QL[5], double QR[5], double *pL, double *pR) {
  const ptrdiff_t s = C->G.s[d];
  const double *const *q = C->q;
  const double *p = C->p;
  ptrdiff_t nm = (C->nv[n0 - s] > BLANKWALL) ? n0 + s : n0 - s;     /* rhs.c:2674-2680 */
  ptrdiff_t np = (C->nv[n0 + 2 * s] > BLANKWALL) ? n0 : n0 + 2 * s; /* rhs.c:2681-2687 */
  for (int a = 0; a < 5; a++) {
    QL[a] = muscl_l(q[a][nm], q[a][n0], q[a][n0 + s]);
    QR[a] = muscl_r(q[a][n0], q[a][n0 + s], q[a][np]);
  }
  *pL = muscl_l(p[nm], p[n0], p[n0 + s]);
  *pR = muscl_r(p[n0], p[n0 + s], p[np]);
}

static void face_metric(const ctx_t *C, int d, ptrdiff_t n0, double h[3]) {
  const double *const *m = C->met[d];
  ptrdiff_t n1 = n0 + C->G.s[d];
  for (int a = 0; a < 3; a++) h[a] = 0.5 * (m[a][n0] + m[a][n1]);
}

/* formConvection face flux (rhs.c:2647-3121), face between n0 and n0+e_d. */
static void conv_face_std(const ctx_t *C, int d, int i, int j, int k, double F[5]) {
  const cbo_config *c = C->c;
  const ptrdiff_t s = C->G.s[d];
  const ptrdiff_t n0 = IX(&C->G, i, j, k), n1 = n0 + s;
  const int pos = d == 0 ? i : d == 1 ? j : k;
  const int m = C->G.m[d];
  const int fo = c->fluxorder;
  const double *nv = C->nv;
  double QL[5], QR[5], pL, pR;
  if (d == 1 && j == 0 && c->isothermal && c->bctype[2] == 1) { /* rhs.c:2822-2827 */
    ld5(C, n0, QL); ld5(C, n0, QR); pL = pR = C->p[n0];
  } else if (d == 1 && j == m - 2 && c->isothermal && c->bctype[3] == 1) { /* rhs.c:2828-2833 */
    ld5(C, n1, QL); ld5(C, n1, QR); pL = pR = C->p[n1];
  } else if (fo == 1 || pos == 0 || pos == m - 2 || (nv[n0] + nv[n1]) > BLANKWALL) {
    ld5(C, n0, QL); ld5(C, n1, QR); pL = C->p[n0]; pR = C->p[n1];
  } else if (fo == 2 || (c->weno_order != 5 && d > 0 && j < 30 && k < 7)) { /* quirk: rhs.c:2840, 2997 */
    recon_muscl(C, d, n0, QL, QR, &pL, &pR);
  } else if (!(c->weno_order == 5 && recon_weno5(C, d, pos, n0, QL, QR, &pL, &pR))) {
    /* ENO fallbacks: xi also requires i+2 < mx (rhs.c:2706); eta/zeta do not */
    int el = nv[n0 - s] > BLANKWALL && (d != 0 || (i + 2) < C->G.m[0]);
    int er = nv[n0 + 2 * s] > BLANKWALL;
    int iso = (d == 1 && j == 1 && c->isothermal && c->bctype[2] == 1);
    recon_weno(C, d, pos, n0, el, er, iso, QL, QR, &pL, &pR);
  }
  double h[3];
  face_metric(C, d, n0, h);
  int use_qr_l = (pos == m - 2 && c->bctype[2 * d + 1] == 1);
  int r_from_l = (pos == 0 && c->bctype[2 * d] == 1);
  if (c->flux == 1) roe(QL, QR, pL, pR, h, use_qr_l, r_from_l, F);
  else rusanov(QL, QR, pL, pR, h, use_qr_l, r_from_l, F);
}

/* formConvectionLES face flux (rhs.c:3466-3705 and its eta/zeta copies). */
static void conv_face_les(const ctx_t *C, int d, int i, int j, int k, const double *const sig[3], double F[5]) {
  const cbo_config *c = C->c;
  const ptrdiff_t s = C->G.s[d];
  const ptrdiff_t n0 = IX(&C->G, i, j, k), n1 = n0 + s;
  const int pos = d == 0 ? i : d == 1 ? j : k;
  const int m = C->G.m[d];
  const double *nv = C->nv;
  const double *const *q = C->q;
  const double *p = C->p;
  double h[3];
  face_metric(C, d, n0, h);
  double sigma = sig[d][n0];

  /* central flux */
  double Fc[5];
  int four = 0;
  if (pos > 0 && pos < m - 2) {
    double nsum;
    if (d == 0) nsum = nv[n0] + nv[n1] + nv[n0 + 2 * s] + nv[n0 - s];
    else nsum = nv[n0 - s] + nv[n0] + nv[n1] + nv[n0 + 2 * s];
    four = nsum < 2.9;
  }
  if (four && (c->central == 2 || c->central == 3)) {
    double r[4], u[4], v[4], w[4], e[4], pc[4], ep[4], U[4];
    const double *const *mn = C->met[d];
    for (int a = -1; a < 3; a++) {
      ptrdiff_t L = n0 + a * s;
      int mm = a + 1;
      r[mm] = q[0][L]; u[mm] = q[1][L]; v[mm] = q[2][L]; w[mm] = q[3][L]; e[mm] = q[4][L];
      pc[mm] = p[L];
      ep[mm] = pc[mm] + e[mm];
      U[mm] = 1. / q[0][L] * (mn[0][L] * q[1][L] + mn[1][L] * q[2][L] + mn[2][L] * q[3][L]);
    }
#define FP2(A, B) ((A[1] + A[2]) * (B[1] + B[2]) / 3.0 - 1. / 24. * (A[0] * B[0] + A[0] * B[2] + A[1] * B[1] + A[1] * B[3] + A[2] * B[2] + A[2] * B[0] + A[3] * B[1] + A[3] * B[3]))
#define FP1(A, B) (1.0 / 12.0 * (-A[0] * B[0] + 7 * A[1] * B[1] + 7 * A[2] * B[2] - A[3] * B[3]))
    double fp4 = 1.0 / 12.0 * (-pc[0] + 7 * pc[1] + 7 * pc[2] - pc[3]); /* rhs.c:2483-2489 */
    if (c->central == 2) { /* rhs.c:2468-2474 */
      Fc[0] = FP2(r, U);
      Fc[1] = FP2(u, U) + fp4 * h[0];
      Fc[2] = FP2(v, U) + fp4 * h[1];
      Fc[3] = FP2(w, U) + fp4 * h[2];
      Fc[4] = FP2(ep, U);
    } else {
      Fc[0] = FP1(r, U);
      Fc[1] = FP1(u, U) + fp4 * h[0];
      Fc[2] = FP1(v, U) + fp4 * h[1];
      Fc[3] = FP1(w, U) + fp4 * h[2];
      Fc[4] = FP1(ep, U);
    }
#undef FP2
#undef FP1
  } else {
    double rc = 0.5 * (q[0][n0] + q[0][n1]);
    double uc = 0.5 * (q[1][n0] + q[1][n1]);
    double vc = 0.5 * (q[2][n0] + q[2][n1]);
    double wc = 0.5 * (q[3][n0] + q[3][n1]);
    double ec = 0.5 * (q[4][n0] + q[4][n1]);
    double Uc = (h[0] * uc + h[1] * vc + h[2] * wc) / rc;
    double pa = 0.5 * (p[n0] + p[n1]);
    Fc[0] = rc * Uc;
    Fc[1] = uc * Uc + pa * h[0];
    Fc[2] = vc * Uc + pa * h[1];
    Fc[3] = wc * Uc + pa * h[2];
    Fc[4] = Uc * (ec + pa);
  }

  /* upwind flux */
  double QL[5], QR[5], pL, pR;
  /* quirk: the zeta test reads nvert[k+1][j][1] (rhs.c:4046) */
  double nsum2 = (d == 2) ? nv[n0] + nv[IX(&C->G, 1, j, k + 1)] : nv[n0] + nv[n1];
  int fo = c->fluxorder;
  if (fo == 1 || ((pos == 0 || pos == m - 2) && c->bctype[2 * d] != 7) || nsum2 > BLANKWALL) {
    ld5(C, n0, QL); ld5(C, n1, QR); pL = p[n0]; pR = p[n1];
  } else if (fo == 2) {
    recon_muscl(C, d, n0, QL, QR, &pL, &pR);
  } else if (!(c->weno_order == 5 && recon_weno5(C, d, pos, n0, QL, QR, &pL, &pR))) {
    int el = nv[n0 - s] > BLANKWALL && (d != 0 || (i + 2) < C->G.m[0]);
    int er = nv[n0 + 2 * s] > BLANKWALL;
    recon_weno(C, d, pos, n0, el, er, 0, QL, QR, &pL, &pR);
  }
  double Fw[5];
  if (c->flux == 1) roe(QL, QR, pL, pR, h, 0, 0, Fw);
  else rusanov(QL, QR, pL, pR, h, 0, 0, Fw);
  for (int a = 0; a < 5; a++) F[a] = Fw[a] * (1.0 - sigma) + Fc[a] * sigma;
}

/* formViscous face flux (rhs.c:1488-2115), face between n0 and n0+e_d.
 * u,v,w: velocity planes; T = p/rho plane.  Fv: 5 values, A: LES stress
 * part (t + Ss) for the energy correction. */
typedef struct {
  const double *u[3];
  const double *T;
  const double *nut;
  const double *const *sig;
  const double *aj;
} visc_t;

static inline int avail_blocked(double v) { return v > SOLID && v < INNERBLANK; }

static void visc_face(const ctx_t *C, const visc_t *V, int d, int i, int j, int k, double Fv[5], double A[3]) {
  const cbo_config *c = C->c;
  const geom *G = &C->G;
  const ptrdiff_t s = G->s[d];
  const ptrdiff_t n0 = IX(G, i, j, k), n1 = n0 + s;
  const int pos = d == 0 ? i : d == 1 ? j : k;
  const int m = G->m[d];
  const double *nv = C->nv;
  /* D[f][e]: derivative of field f (u, v, w, T) along computational dir e */
  double D[4][3];
  const double *fld[4] = {V->u[0], V->u[1], V->u[2], V->T};
  for (int f = 0; f < 4; f++) D[f][d] = fld[f][n1] - fld[f][n0];
  for (int e = 0; e < 3; e++) {
    if (e == d) continue;
    ptrdiff_t t = G->s[e];
    int plus_blocked = avail_blocked(nv[n0 + t]) || avail_blocked(nv[n1 + t]);
    int minus_blocked = avail_blocked(nv[n0 - t]) || avail_blocked(nv[n1 - t]);
    for (int f = 0; f < 4; f++) {
      const double *x = fld[f];
      if (plus_blocked) {
        if (f == 3 && d == 0 && e == 2) /* quirk: dpdz typo, rhs.c:1544-1545 */
          D[f][e] = (x[n1] + x[n0] - x[n1 - t] - x[n0]) * 0.5;
        else
          D[f][e] = (x[n1] + x[n0] - x[n1 - t] - x[n0 - t]) * 0.5;
      } else if (minus_blocked) {
        D[f][e] = (x[n1 + t] + x[n0 + t] - x[n1] - x[n0]) * 0.5;
      } else {
        D[f][e] = (x[n1 + t] + x[n0 + t] - x[n1 - t] - x[n0 - t]) * 0.25;
      }
    }
  }
  double dudc = D[0][0], dude = D[0][1], dudz = D[0][2];
  double dvdc = D[1][0], dvde = D[1][1], dvdz = D[1][2];
  double dwdc = D[2][0], dwde = D[2][1], dwdz = D[2][2];
  double dpdc = D[3][0], dpde = D[3][1], dpdz = D[3][2];

  double mh[3][3]; /* face metrics: mh[0]=csi, mh[1]=eta, mh[2]=zet */
  for (int e = 0; e < 3; e++)
    for (int a = 0; a < 3; a++) mh[e][a] = 0.5 * (C->met[e][a][n0] + C->met[e][a][n1]);
  const double *md = mh[d];
  double csi0 = mh[0][0], csi1 = mh[0][1], csi2 = mh[0][2];
  double eta0 = mh[1][0], eta1 = mh[1][1], eta2 = mh[1][2];
  double zet0 = mh[2][0], zet1 = mh[2][1], zet2 = mh[2][2];
  double g11 = mh[0][0] * md[0] + mh[0][1] * md[1] + mh[0][2] * md[2];
  double g21 = mh[1][0] * md[0] + mh[1][1] * md[1] + mh[1][2] * md[2];
  double g31 = mh[2][0] * md[0] + mh[2][1] * md[1] + mh[2][2] * md[2];

  double r11 = dudc * csi0 + dude * eta0 + dudz * zet0;
  double r21 = dvdc * csi0 + dvde * eta0 + dvdz * zet0;
  double r31 = dwdc * csi0 + dwde * eta0 + dwdz * zet0;
  double r12 = dudc * csi1 + dude * eta1 + dudz * zet1;
  double r22 = dvdc * csi1 + dvde * eta1 + dvdz * zet1;
  double r32 = dwdc * csi1 + dwde * eta1 + dwdz * zet1;
  double r13 = dudc * csi2 + dude * eta2 + dudz * zet2;
  double r23 = dvdc * csi2 + dvde * eta2 + dvdz * zet2;
  double r33 = dwdc * csi2 + dwde * eta2 + dwdz * zet2;

  double ajc = 0.5 * (V->aj[n0] + V->aj[n1]);
  double nu = 1. / c->ren;
  if (c->les) {
    /* quirk: eta and zeta faces average rho over i and i+1 (rhs.c:1835, 2034) */
    ptrdiff_t nr = (d == 0) ? n1 : n0 + G->s[0];
    nu = 1. / c->ren * 0.5 * (C->q[0][n0] + C->q[0][nr]);
  }
  if (c->visT) { /* Sutherland's law on the face temperature (rhs.c:1627-1637, 1837-1846, 2036-2045) */
    const double C_sutherland = 110.4; /* rhs.c:1410 */
    const double Tr = c->gamma * c->ma * c->ma * (C->p[n0] + C->p[n1]) / (C->q[0][n0] + C->q[0][n1]);
    if (Tr < 0) nu = 1. / c->ren;
    else nu = 1. / c->ren * (1 + C_sutherland / c->tref) / (Tr + C_sutherland / c->tref) * pow(Tr, 1.5);
  }
  double div = 2. / 3. * (dudc * csi0 + dude * eta0 + dudz * zet0 + dvdc * csi1 + dvde * eta1 + dvdz * zet1 +
                          dwdc * csi2 + dwde * eta2 + dwdz * zet2);

  Fv[0] = 0.;
  Fv[1] = (g11 * dudc + g21 * dude + g31 * dudz + r11 * md[0] + r21 * md[1] + r31 * md[2]) * ajc * (nu);
  Fv[2] = (g11 * dvdc + g21 * dvde + g31 * dvdz + r12 * md[0] + r22 * md[1] + r32 * md[2]) * ajc * (nu);
  Fv[3] = (g11 * dwdc + g21 * dwde + g31 * dwdz + r13 * md[0] + r23 * md[1] + r33 * md[2]) * ajc * (nu);
  Fv[1] -= div * md[0] * ajc * nu;
  Fv[2] -= div * md[1] * ajc * nu;
  Fv[3] -= div * md[2] * ajc * nu;

  double uh[3];
  if (pos == 0 && c->bctype[2 * d] == 1) {
    for (int a = 0; a < 3; a++) uh[a] = V->u[a][n0];
  } else if (pos == m - 2 && c->bctype[2 * d + 1] == 1) {
    for (int a = 0; a < 3; a++) uh[a] = V->u[a][n1];
  } else {
    for (int a = 0; a < 3; a++) uh[a] = 0.5 * (V->u[a][n1] + V->u[a][n0]);
  }
  double gm = c->gamma;
  Fv[4] = (Fv[1] * uh[0] + Fv[2] * uh[1] + Fv[3] * uh[2]) +
          (g11 * dpdc + g21 * dpde + g31 * dpdz) * ajc * (gm * nu / c->pr / (gm - 1.0));

  A[0] = A[1] = A[2] = 0.;
  if (c->les) { /* rhs.c:1677-1710 */
    double nut = 0.5 * (V->nut[n0] * V->sig[d][n0] + V->nut[n1] * V->sig[d][n1]);
    double rho_c = 0.5 * (C->q[0][n0] + C->q[0][n1]);
    double sigma_c = 0.5 * (V->sig[d][n0] + V->sig[d][n1]);
    if ((c->bctype[2 * d] == 1 && pos == 0) || (c->bctype[2 * d + 1] == 1 && pos == m - 2)) nut = 0;
    double tx = (g11 * dudc + g21 * dude + g31 * dudz + r11 * md[0] + r21 * md[1] + r31 * md[2] - div * md[0]) * ajc * (nut * rho_c);
    double ty = (g11 * dvdc + g21 * dvde + g31 * dvdz + r12 * md[0] + r22 * md[1] + r32 * md[2] - div * md[1]) * ajc * (nut * rho_c);
    double tz = (g11 * dwdc + g21 * dwde + g31 * dwdz + r13 * md[0] + r23 * md[1] + r33 * md[2] - div * md[2]) * ajc * (nut * rho_c);
    double S2 = .5 * ((r11 - div) * (r11 - div) + r12 * r12 + r13 * r13 + r21 * r21 + (r22 - div) * (r22 - div) +
                      r23 * r23 + r31 * r31 + r32 * r32 + (r33 - div) * (r33 - div));
    double filter = pow(1. / V->aj[n0], 1. / 3.);
    double pf = pow(filter, 2.0);
    double ssx = -S2 * pf * c->ci * 2.0 / 3.0 * md[0] * rho_c * sigma_c;
    double ssy = -S2 * pf * c->ci * 2.0 / 3.0 * md[1] * rho_c * sigma_c;
    double ssz = -S2 * pf * c->ci * 2.0 / 3.0 * md[2] * rho_c * sigma_c;
    Fv[1] += tx + ssx;
    Fv[2] += ty + ssy;
    Fv[3] += tz + ssz;
    A[0] = tx + ssx;
    A[1] = ty + ssy;
    A[2] = tz + ssz;
  }
}

/* ------------------------------------------------------------------------ */
/* formRHS  (rhs.c:4703-4736) with MultAj (rhs.c:4575-4701)                  */
/* ------------------------------------------------------------------------ */
/* lp_in: the local pressure lP the reference reads (NULL: EqOfState of q). */
static int rhs_impl(const cbo_config *c, const double *const q[5], const double *lp_in, const double *const csi[3],
                    const double *const eta[3], const double *const zet[3], const double *aj,
                    const double *nvert, const double *nut, const double *const sig[3],
                    double *const rhs[5]) {
  geom G = mkgeom(c);
  const int mx = G.m[0], my = G.m[1], mz = G.m[2];
  if (mx < 5 || my < 5 || mz < 5) return 3;
  if (c->les && (!nut || !sig)) return 4;
  double *p = (double *)malloc(G.n * sizeof(double));
  if (lp_in) memcpy(p, lp_in, G.n * sizeof(double));
  else cbo_eos(c, q, p);
  ctx_t C;
  C.c = c; C.G = G; C.q = q; C.p = p; C.nv = nvert;
  C.met[0] = csi; C.met[1] = eta; C.met[2] = zet;

  /* face buffers: Fc[d][5], Fv[d][5], Al[d][3] */
  double *buf = (double *)calloc(G.n * 39, sizeof(double));
  double *Fc[3][5], *Fv[3][5], *Al[3][3];
  for (int d = 0; d < 3; d++) {
    for (int a = 0; a < 5; a++) { Fc[d][a] = buf + G.n * (d * 13 + a); Fv[d][a] = buf + G.n * (d * 13 + 5 + a); }
    for (int a = 0; a < 3; a++) Al[d][a] = buf + G.n * (d * 13 + 10 + a);
  }

  /* face ranges: along d from 0 to m-2, transverse interior (rhs.c:2647 etc.);
   * -twoD 1 computes no i-faces, whose fluxes stay zero (rhs.c:2646, 3465) */
  for (int d = 0; d < 3; d++) {
    if (d == 0 && c->twod == 1) continue;
    int lo[3] = {1, 1, 1}, hi[3] = {mx - 1, my - 1, mz - 1};
    lo[d] = 0;
    for (int k = lo[2]; k < hi[2]; k++)
      for (int j = lo[1]; j < hi[1]; j++)
        for (int i = lo[0]; i < hi[0]; i++) {
          double F[5];
          if (c->les) conv_face_les(&C, d, i, j, k, sig, F);
          else conv_face_std(&C, d, i, j, k, F);
          ptrdiff_t n = IX(&G, i, j, k);
          for (int a = 0; a < 5; a++) Fc[d][a][n] = F[a];
        }
  }

  double *ucat = NULL;
  visc_t V;
  if (!c->inviscid) {
    /* CalcUCat (rhs.c:1322-1365) over the ghosted box; T = p/rho */
    ucat = (double *)malloc(G.n * 4 * sizeof(double));
    for (size_t n = 0; n < G.n; n++) {
      double r = q[0][n];
      ucat[n] = (r != 0.0 && c->twod != 1) ? q[1][n] / r : 0.0; /* x zero with -twoD 1 (rhs.c:1349) */
      ucat[G.n + n] = r != 0.0 ? q[2][n] / r : 0.0;
      ucat[2 * G.n + n] = r != 0.0 ? q[3][n] / r : 0.0;
      ucat[3 * G.n + n] = r != 0.0 ? p[n] / r : 0.0;
    }
    V.u[0] = ucat; V.u[1] = ucat + G.n; V.u[2] = ucat + 2 * G.n; V.T = ucat + 3 * G.n;
    V.nut = nut; V.sig = sig; V.aj = aj;
    for (int d = 0; d < 3; d++) {
      if (d == 0 && c->twod == 1) continue; /* rhs.c:1487 */
      int lo[3] = {1, 1, 1}, hi[3] = {mx - 1, my - 1, mz - 1};
      lo[d] = 0;
      for (int k = lo[2]; k < hi[2]; k++)
        for (int j = lo[1]; j < hi[1]; j++)
          for (int i = lo[0]; i < hi[0]; i++) {
            double F[5], A[3];
            visc_face(&C, &V, d, i, j, k, F, A);
            ptrdiff_t n = IX(&G, i, j, k);
            for (int a = 0; a < 5; a++) Fv[d][a][n] = F[a];
            for (int a = 0; a < 3; a++) Al[d][a][n] = A[a];
          }
    }
  }

  for (int a = 0; a < 5; a++) memset(rhs[a], 0, G.n * sizeof(double));
  const ptrdiff_t si = G.s[0], sj = G.s[1], sk = G.s[2];
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        double conv[5] = {0, 0, 0, 0, 0}, visc[5] = {0, 0, 0, 0, 0};
        if (nvert[n] < BLANK) { /* rhs.c:3159-3205 / 4205-4246 */
          for (int a = 0; a < 5; a++)
            conv[a] = Fc[0][a][n] - Fc[0][a][n - si] + Fc[1][a][n] - Fc[1][a][n - sj] + Fc[2][a][n] - Fc[2][a][n - sk];
          if (c->twod == 1) conv[1] = 0.; /* rhs.c:3168-3173, 4215-4220 */
          if (c->les) {
            conv[3] = conv[3] - c->ratio / aj[n] * q[0][n] / c->dt;
            conv[4] = conv[4] - c->ratio / aj[n] * q[3][n] / c->dt;
          }
        }
        if (!c->inviscid) { /* rhs.c:2123-2199 */
          for (int a = 1; a < 5; a++)
            visc[a] = Fv[0][a][n] - Fv[0][a][n - si] + Fv[1][a][n] - Fv[1][a][n - sj] + Fv[2][a][n] - Fv[2][a][n - sk];
          if (c->twod == 1) visc[1] = 0.; /* rhs.c:2135-2140 */
          if (c->les && j > 2 && j < my - 2 && nvert[n] < 0.5) {
            double rL = (q[0][n] + q[0][n - si]) * 0.5, rR = (q[0][n + si] + q[0][n]) * 0.5;
            double rD = (q[0][n] + q[0][n - sj]) * 0.5, rU = (q[0][n + sj] + q[0][n]) * 0.5;
            double rB = (q[0][n] + q[0][n - sk]) * 0.5, rF = (q[0][n + sk] + q[0][n]) * 0.5;
            double u0 = q[1][n] / q[0][n], u1 = q[2][n] / q[0][n], u2 = q[3][n] / q[0][n];
            double e = 0;
            double uu[3] = {u0, u1, u2};
            for (int a = 0; a < 3; a++) {
              double t = rR * Al[0][a][n] - rL * Al[0][a][n - si] + rU * Al[1][a][n] - rD * Al[1][a][n - sj] +
                         rF * Al[2][a][n] - rB * Al[2][a][n - sk];
              e = (a == 0) ? uu[a] * t : e + uu[a] * t;
            }
            visc[4] += e;
          }
        }
        for (int a = 0; a < 5; a++) {
          double r = visc[a] - conv[a]; /* VecWAXPY(Rhs, -1, Conv, Visc) */
          rhs[a][n] = (nvert[n] < BLANK) ? r * aj[n] : 0.; /* MultAj */
        }
      }
  free(ucat);
  free(buf);
  free(p);
  return 0;
}

int cbo_rhs(const cbo_config *c, const double *const q[5], const double *const csi[3],
            const double *const eta[3], const double *const zet[3], const double *aj,
            const double *nvert, const double *nut, const double *const sig[3],
            double *const rhs[5]) {
  return rhs_impl(c, q, NULL, csi, eta, zet, aj, nvert, nut, sig, rhs);
}

int cbo_rhs_lp(const cbo_config *c, const double *const q[5], const double *lp, const double *const csi[3],
               const double *const eta[3], const double *const zet[3], const double *aj,
               const double *nvert, const double *nut, const double *const sig[3],
               double *const rhs[5]) {
  return rhs_impl(c, q, lp, csi, eta, zet, aj, nvert, nut, sig, rhs);
}

/* ------------------------------------------------------------------------ */
/* Compute_eddy_viscosity_LES  (les.c:1477-1574), constant CS (les.c:135-150) */
/* ------------------------------------------------------------------------ */
void cbo_eddy_viscosity(const cbo_config *c, const double *const qu[5], const double *const csi[3],
                        const double *const eta[3], const double *const zet[3], const double *aj,
                        const double *nvert, double *nut) {
  geom G = mkgeom(c);
  const ptrdiff_t si = G.s[0], sj = G.s[1], sk = G.s[2];
  for (int k = 1; k < G.m[2] - 1; k++)
    for (int j = 1; j < G.m[1] - 1; j++)
      for (int i = 1; i < G.m[0] - 1; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        if (nvert[n] > 0.1) { nut[n] = 0; continue; }
        double d[3][3]; /* d[comp][dir] central differences of velocity */
        for (int a = 0; a < 3; a++) {
          /* lUcat x is zero with -twoD 1 (CalcUCat rhs.c:1349) */
          if (!qu || (a == 0 && c->twod == 1)) { d[a][0] = d[a][1] = d[a][2] = 0.0; continue; }
          const double *r = qu[0], *m = qu[1 + a];
          d[a][0] = (m[n + si] / r[n + si] - m[n - si] / r[n - si]) * 0.5;
          d[a][1] = (m[n + sj] / r[n + sj] - m[n - sj] / r[n - sj]) * 0.5;
          d[a][2] = (m[n + sk] / r[n + sk] - m[n - sk] / r[n - sk]) * 0.5;
        }
        double ajc = aj[n];
        double c0 = csi[0][n], c1 = csi[1][n], c2 = csi[2][n];
        double e0 = eta[0][n], e1 = eta[1][n], e2 = eta[2][n];
        double z0 = zet[0][n], z1 = zet[1][n], z2 = zet[2][n];
        double g[3][3]; /* g[comp][x] = d u_comp / d x */
        for (int a = 0; a < 3; a++) {
          g[a][0] = (d[a][0] * c0 + d[a][1] * e0 + d[a][2] * z0) * ajc;
          g[a][1] = (d[a][0] * c1 + d[a][1] * e1 + d[a][2] * z1) * ajc;
          g[a][2] = (d[a][0] * c2 + d[a][1] * e2 + d[a][2] * z2) * ajc;
        }
        double du_dx = g[0][0], du_dy = g[0][1], du_dz = g[0][2];
        double dv_dx = g[1][0], dv_dy = g[1][1], dv_dz = g[1][2];
        double dw_dx = g[2][0], dw_dy = g[2][1], dw_dz = g[2][2];
        double Sdd = 2. / 3. * (du_dx + dv_dy + dw_dz);
        double Sxx = 0.5 * (du_dx + du_dx) - Sdd, Sxy = 0.5 * (du_dy + dv_dx), Sxz = 0.5 * (du_dz + dw_dx);
        double Syx = Sxy, Syy = 0.5 * (dv_dy + dv_dy) - Sdd, Syz = 0.5 * (dv_dz + dw_dy);
        double Szx = Sxz, Szy = Syz, Szz = 0.5 * (dw_dz + dw_dz) - Sdd;
        double Sabs = sqrt(2.0 * (Sxx * Sxx + Sxy * Sxy + Sxz * Sxz + Syx * Syx + Syy * Syy + Syz * Syz +
                                  Szx * Szx + Szy * Szy + Szz * Szz));
        double filter = pow(1. / aj[n], 1. / 3.);
        nut[n] = c->cs_const * pow(filter, 2.0) * Sabs;
      }
  cbo_fill_ghosts(c, nut);
}

/* ------------------------------------------------------------------------ */
/* RungeKutta stage combine  (solvers.c:232-271)                             */
/* ------------------------------------------------------------------------ */
void cbo_rk_combine(const cbo_config *c, int istage, const double *const qold[5],
                    const double *const qin[5], const double *const rhs[5], double *const qout[5]) {
  geom G = mkgeom(c);
  double alfa[3] = {1., 1 / 4., 2 / 3.}, beta[3] = {1., 3 / 4., 1 / 3.};
  if (c->fluxorder < 3) { alfa[1] = 1 / 2.; beta[1] = 1 / 2.; }
  double adt = alfa[istage] * c->dt * c->st;
  for (int k = 0; k < G.m[2]; k++)
    for (int j = 0; j < G.m[1]; j++)
      for (int i = 0; i < G.m[0]; i++) {
        ptrdiff_t n = IX(&G, i, j, k);
        for (int a = 0; a < 5; a++) {
          if (istage == 0) qout[a][n] = qold[a][n] + adt * rhs[a][n];               /* VecWAXPY */
          else qout[a][n] = beta[istage] * qold[a][n] + adt * rhs[a][n] + alfa[istage] * qin[a][n]; /* VecAXPBYPCZ */
        }
      }
}

/* ------------------------------------------------------------------------ */
/* FormBCS periodic part  (rhs.c:1107-1227, then rhs.c:1305-1308)            */
/* qin is the ghosted local state of the stage input: FormBCS reads lQ before */
/* it is refreshed, so boundary nodes receive the previous stage's values.   */
/* ------------------------------------------------------------------------ */
int cbo_bc_periodic(const cbo_config *c, const double *const qin[5], double *const qout[5]) {
  geom G = mkgeom(c);
  const int mx = G.m[0], my = G.m[1], mz = G.m[2];
  for (int b = 0; b < 6; b++) if (c->bctype[b] != 7) return 5; /* non-periodic BCs: not restated */
  const ptrdiff_t si = G.s[0], sj = G.s[1], sk = G.s[2];
  /* i faces: guard k>0 && k<KM && j>0 && j<JM with KM = mz, JM = my */
  for (int k = 1; k < mz; k++)
    for (int j = 1; j < my; j++) {
      ptrdiff_t n = IX(&G, 0, j, k);
      for (int a = 0; a < 5; a++) qout[a][n] = qin[a][n - 2 * si];
      n = IX(&G, mx - 1, j, k);
      for (int a = 0; a < 5; a++) qout[a][n] = qin[a][n + 2 * si];
    }
  /* j faces: j=0 for k>0; j=my-1 for k in [1, mz-2] */
  for (int k = 1; k < mz; k++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, 0, k);
      for (int a = 0; a < 5; a++) qout[a][n] = qin[a][n - 2 * sj];
    }
  for (int k = 1; k < mz - 1; k++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, my - 1, k);
      for (int a = 0; a < 5; a++) qout[a][n] = qin[a][n + 2 * sj];
    }
  /* k faces: unguarded */
  for (int j = 0; j < my; j++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, j, 0);
      for (int a = 0; a < 5; a++) qout[a][n] = qin[a][n - 2 * sk];
      n = IX(&G, i, j, mz - 1);
      for (int a = 0; a < 5; a++) qout[a][n] = qin[a][n + 2 * sk];
    }
  for (int a = 0; a < 5; a++) cbo_fill_ghosts(c, qout[a]);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* FormBCS  (rhs.c:477-1227)                                                 */
/* q: the stage output, every node already combined by the RK update; lq:    */
/* the stale ghosted stage input (its pressure lp from the EOS); qold: the   */
/* step's initial state.  Face order i, j, k, then the periodic copies, then */
/* the wrap of periodic directions (DMGlobalToLocal).  Codes: i 3, 51; j 3,   */
/* 10, 1 (isothermal 0/1/2); k-lo 3, 52, 55, 44, 45, 51, 10, 47; k-hi 3,    */
/* 44, 45, 49, 51, 10, 8; 7 periodic; any other code leaves the face as the  */
/* RK update left it, as in the reference.  52 and 47 read the node          */
/* coordinates (c->coor_x/coor_y; 5 is returned without them) and 47 the     */
/* step index ti.                                                            */
/* ------------------------------------------------------------------------ */
/* lp_in: the local pressure lP (NULL: EqOfState of lq); p (may be NULL): the
 * global P, which receives the periodic copies and then the ghost wrap. */
static int nvert_ok(const double *nv, ptrdiff_t n) { return !nv || nv[n] < 1.5; }

static int formbcs_impl(const cbo_config *c, int ti, double alfa, const double *const lq[5], const double *lp_in,
                        const double *const qold[5], const double *const eta[3], const double *const zet[3],
                        const double *aj, const double *nvert_in, double *const q[5], double *p) {
  geom G = mkgeom(c);
  const int mx = G.m[0], my = G.m[1], mz = G.m[2];
  const int *bc = c->bctype;
  if ((bc[4] == 52 || bc[4] == 47) && (!c->coor_x || !c->coor_y)) return 5;
  if ((bc[0] == 7) != (bc[1] == 7) || (bc[2] == 7) != (bc[3] == 7) || (bc[4] == 7) != (bc[5] == 7)) return 5;
  const ptrdiff_t si = G.s[0], sj = G.s[1], sk = G.s[2];
  const double g = c->gamma, Ma = c->ma;
  double *lp = (double *)malloc(G.n * sizeof(double));
  if (lp_in) memcpy(lp, lp_in, G.n * sizeof(double));
  else cbo_eos(c, lq, lp);
#define RO(n) q[0][n]
#define RU(n) q[1][n]
#define RV(n) q[2][n]
#define RW(n) q[3][n]
#define RE(n) q[4][n]
  /* i BC (rhs.c:601-636) */
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++) {
      ptrdiff_t n = IX(&G, 0, j, k);
      if (bc[0] == 3) {
        RO(n) = RO(n + si); RU(n) = 0.; RV(n) = RV(n + si); RW(n) = RW(n + si); RE(n) = RE(n + si);
      } else if (bc[0] == 51) {
        RO(n) = 0.445; RU(n) = 0.311; RV(n) = 0.; RW(n) = 0.; RE(n) = 8.928;
      }
      n = IX(&G, mx - 1, j, k);
      if (bc[1] == 3) {
        RO(n) = RO(n - si); RU(n) = 0.; RV(n) = RV(n - si); RW(n) = RW(n - si); RE(n) = RE(n - si);
      } else if (bc[0] == 51) { /* quirk: the high-i Lax state is keyed on bctype[0] (rhs.c:627) */
        RO(n) = 0.5; RU(n) = 0.; RV(n) = 0.; RW(n) = 0.; RE(n) = 1.4275;
      }
    }
  /* j BC (rhs.c:639-835) */
  for (int k = 0; k < mz; k++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, 0, k);
      if (bc[2] == 3) {
        RO(n) = RO(n + sj); RU(n) = RU(n + sj); RV(n) = 0.; RW(n) = RW(n + sj); RE(n) = RE(n + sj);
      } else if (bc[2] == 10) {
        RO(n) = RO(n + sj); RU(n) = 0.; RV(n) = RV(n + sj); RW(n) = RW(n + sj); RE(n) = RE(n + sj);
      } else if (bc[2] == 1) {
        RU(n) = 0.0; RV(n) = 0.0; RW(n) = 0.0;
        if (c->isothermal == 2 && alfa != 0 && nvert_ok(nvert_in, n)) {
          /* characteristic isothermal wall (Poinsot & Lele), one pass (rhs.c:663-733, itr_tmp 1) */
          const double a_sound = sqrt(c->twall / (Ma * Ma));
          const double beta = sqrt(eta[1][n] * eta[1][n] + eta[0][n] * eta[0][n] + eta[2][n] * eta[2][n]);
          const double L0 = -a_sound * beta;
          if (!(k == 0 || k == mz - 1)) {
            const ptrdiff_t n1 = n + sj, n2 = n + 2 * sj;
            double L = L0 * aj[n] *
                       ((-0.5 * lp[n2] + 2 * lp[n1] - 1.5 * lp[n]) -
                        lq[0][n] * a_sound / beta *
                            (eta[1][n] * (-0.5 * lq[2][n2] / lq[0][n2] + 2. * lq[2][n1] / lq[0][n1] - 1.5 * lq[2][n] / lq[0][n]) +
                             eta[2][n] * (-0.5 * lq[3][n2] / lq[0][n2] + 2. * lq[3][n1] / lq[0][n1] - 1.5 * lq[3][n] / lq[0][n])));
            if (c->twod != 1)
              L -= L0 * aj[n] * lq[0][n] * a_sound / beta * eta[0][n] *
                   (-0.5 * lq[1][n2] / lq[0][n2] + 2. * lq[1][n1] / lq[0][n1] - 1.5 * lq[1][n] / lq[0][n]);
            RO(n) = qold[0][n] - c->dt * alfa * L / a_sound / a_sound;
            lp[n] = RO(n) * c->twall / (g * Ma * Ma);
          }
        } else {
          lp[n] = lp[n + sj];
          RO(n) = lp[n] * (g * Ma * Ma);
          RE(n) = lp[n] / (g - 1);
        }
      }
      n = IX(&G, i, my - 1, k);
      if (bc[3] == 3) {
        RO(n) = RO(n - sj); RU(n) = RU(n - sj); RV(n) = 0.; RW(n) = RW(n - sj); RE(n) = RE(n - sj);
      } else if (bc[3] == 10) {
        RO(n) = RO(n - sj); RU(n) = 0.; RV(n) = RV(n - sj); RW(n) = RW(n - sj); RE(n) = RE(n - sj);
      } else if (bc[3] == 1) {
        RU(n) = 0.0; RV(n) = 0.0; RW(n) = 0.0;
        if (c->isothermal == 2) { /* rhs.c:803-818 */
          const ptrdiff_t m1 = n - sj, m2 = n - 2 * sj;
          const double a_sound = sqrt(g * lp[m1] / lq[0][m1]);
          const double L0 = lq[2][m1] / lq[0][m1] - a_sound;
          double L;
          if (k == 0 || k == mz - 1 || L0 > 0.) L = 0.;
          else
            L = L0 * aj[m1] * eta[1][m1] *
                ((lp[m1] - lp[m2]) - lq[0][m1] * a_sound * (lq[2][n] / lq[0][n] - lq[2][m1] / lq[0][m1]));
          RO(n) = qold[0][n] - c->dt * alfa * L / a_sound / a_sound;
          lp[n] = RO(n) * c->twall / (g * Ma * Ma);
        } else if (c->isothermal == 1) {
          RO(n) = lp[n] * (g * Ma * Ma);
          lp[n] = lp[n - sj];
        } else {
          RO(n) = RO(n - sj);
          lp[n] = lp[n - sj];
        }
        RE(n) = lp[n] / (g - 1.0);
      }
    }
  /* k BC (rhs.c:840-1087) */
  const int ls = (bc[2] == 1) ? 1 : 0, le = (bc[3] == 1) ? my - 1 : my;
  const double u55 = Ma, rho55 = g;
  for (int j = ls; j < le; j++)
    for (int i = 0; i < mx; i++) {
      ptrdiff_t n = IX(&G, i, j, 0);
      if (bc[4] == 3) {
        RO(n) = RO(n + sk); RU(n) = RU(n + sk); RV(n) = RV(n + sk); RW(n) = 0.; RE(n) = RE(n + sk);
      } else if (bc[4] == 55) {
        RO(n) = rho55; RW(n) = rho55 * u55; RE(n) = 0.5 * rho55 * u55 * u55 + 1. / (g - 1.);
      } else if (bc[4] == 44) {
        RO(n) = RO(n + sk); RU(n) = 0.; RV(n) = 0.; RW(n) = RW(n + sk); RE(n) = RE(n + sk);
      } else if (bc[4] == 45) {
        RO(n) = 1.; RW(n) = 1.; RE(n) = .5 + 1. / (Ma * Ma * g * (g - 1.));
      } else if (bc[4] == 51) {
        RO(n) = 0.445; RW(n) = 0.311; RE(n) = 8.928;
      } else if (bc[4] == 10) {
        RO(n) = 1.; RU(n) = 0.; RV(n) = 0.; RW(n) = 1.; RE(n) = 1. / 0.4 + 0.5;
      } else if (bc[4] == 52) {
        /* characteristic inlet imposing w = cos^2(pi/2 (y - 1)) (rhs.c:854-874);
         * pi is FormBCS's own truncated value (rhs.c:488) */
        const double pi = 3.14159265;
        const ptrdiff_t n1 = n + sk, n2 = n + 2 * sk;
        const double yy = c->coor_y[n];
        const double AA = cos(pi / 2 * (yy - 1.)) * cos(pi / 2 * (yy - 1.));
        const double a_sound = sqrt(g * lp[n1] / lq[0][n1]);
        const double Lam0 = lq[3][n1] / lq[0][n1] - a_sound;
        const double L0 = Lam0 * aj[n1] * zet[2][n1] * ((lp[n2] - lp[n1]) - lq[0][n1] * a_sound * (lq[3][n1] / lq[0][n1] - AA));
        const double L1 = (g - 1.) * L0, L4 = L0;
        const double d0 = 1. / (a_sound * a_sound) * (L1 + 0.5 * (L4 + L0));
        RO(n) = qold[0][n] - c->dt * alfa * d0;
        lp[n] = RO(n) / (g * Ma * Ma);
        RW(n) = RO(n) * AA;
        RU(n) = 0.;
        RV(n) = 0.;
        RE(n) = 0.5 * RW(n) * RW(n) / RO(n) + lp[n] / (g - 1);
      } else if (bc[4] == 47) {
        /* power-law inflow with travelling perturbations in x and time
         * (rhs.c:904-950): below y = 8 w = (y/8)^0.1428 plus a near-wall
         * mode (u is left as the RK update left it), above w = 1, u = 0 plus
         * three modes; rho = 1 */
        const double pi = 3.141592;
        const double c1 = 0.03, c2 = -0.0032, c3 = 0.02, c4 = -0.01, yp1 = 1.0, yp2 = 1.5, yp3 = 2.0;
        const double w0 = 0.1, w1 = 0.25, w2 = 0.125, w3 = 0.0625;
        const double phi1 = 0.0, phi2 = 0.1, phi3 = 0.15, b0 = 0.5 * pi, b1 = 0.75 * pi, b2 = 0.5 * pi, b3 = 0.25 * pi;
        const double yy = c->coor_y[n], xx = c->coor_x[n];
        const double yplus = yy * 0.065 * c->ren;
        if (yy < 8.0) {
          RW(n) = pow(yy / 8.0, 0.1428);
        } else {
          RW(n) = 1.0;
          RU(n) = 0.0;
        }
        if (yy < 8.0) {
          RW(n) += c1 * yplus * exp(-yplus / 12.5) * sin(w0 * ti * c->dt) * cos(b0 * xx);
          RV(n) = c2 * yplus * yplus * exp(-yplus * yplus / 12.5 / 12.5) * sin(w0 * ti * c->dt) * cos(b0 * xx);
        } else if (yy >= 8.0) {
          RW(n) += c3 * yy / yp1 * exp(-yy / yp1) * sin(w1 * ti * c->dt) * cos(b1 * xx + phi1) +
                   c3 * yy / yp2 * exp(-yy / yp2) * sin(w2 * ti * c->dt) * cos(b2 * xx + phi2) +
                   c3 * yy / yp3 * exp(-yy / yp3) * sin(w3 * ti * c->dt) * cos(b3 * xx + phi3);
          RV(n) = c4 * yy * yy / yp1 / yp1 * exp(-yy * yy / yp1 / yp1) * sin(w1 * ti * c->dt) * cos(b1 * xx + phi1) +
                  c4 * yy * yy / yp2 / yp2 * exp(-yy * yy / yp2 / yp2) * sin(w2 * ti * c->dt) * cos(b2 * xx + phi2) +
                  c4 * yy * yy / yp3 / yp3 * exp(-yy * yy / yp3 / yp3) * sin(w3 * ti * c->dt) * cos(b3 * xx + phi3);
        }
        RO(n) = 1.0;
        RE(n) = 0.5 * RW(n) * RW(n) + 1. / (Ma * Ma * g * (g - 1.));
      }
      n = IX(&G, i, j, mz - 1);
      const ptrdiff_t m1 = n - sk, m2 = n - 2 * sk;
      if (bc[5] == 3) {
        RO(n) = RO(m1); RU(n) = RU(m1); RV(n) = RV(m1); RW(n) = 0.; RE(n) = RE(m1);
      } else if (bc[5] == 44) {
        RO(n) = RO(m1); RU(n) = 0.; RV(n) = 0.; RW(n) = RW(m1); RE(n) = RE(m1);
      } else if (bc[5] == 45) {
        RO(n) = RO(m1); RU(n) = RU(m1); RV(n) = RV(m1); RW(n) = RW(m1); RE(n) = RE(m1);
      } else if (bc[5] == 49) { /* characteristic (rhs.c:1003-1042) */
        double Vn, Rplus, Rminus, lambda1, lambda2, sv, pOverrho, pp, a_sound;
        Vn = RW(m1) / RO(m1);
        a_sound = sqrt(g * lp[m1] / RO(m1));
        lambda1 = Vn + a_sound;
        lambda2 = Vn - a_sound;
        if (Vn < 0.) {
          if (lambda1 < 0) {
            RU(n) = 0.; RV(n) = 0.;
            Rplus = Vn + 2 / Ma / (g - 1.);
            Rminus = Vn - 2 / Ma / (g - 1.);
            sv = 1. / (Ma * Ma * g);
          } else {
            Rplus = Vn + 2 * a_sound / (g - 1.);
            Rminus = Vn - 2 / Ma / (g - 1.);
            RU(n) = 0.; RV(n) = 0.;
            sv = 1. / (Ma * Ma * g);
          }
        } else {
          if (lambda2 >= 0) {
            Rplus = Vn + 2 * a_sound / (g - 1.);
            Rminus = Vn - 2 * a_sound / (g - 1.);
            RU(n) = RU(m1);
            RV(n) = RO(m1); /* quirk: rhoV takes rho (rhs.c:1022) */
            sv = lp[m1] / pow(RO(m1), g);
          } else {
            Rminus = Vn - 2 / Ma / (g - 1.);
            Rplus = Vn + 2 * a_sound / (g - 1.);
            RU(n) = RU(m1); RV(n) = RV(m1);
            sv = lp[m1] / pow(RO(m1), g);
          }
        }
        Vn = 0.5 * (Rplus + Rminus);
        a_sound = 0.25 * (g - 1.) * (Rplus - Rminus);
        pOverrho = a_sound * a_sound / (g);
        RO(n) = pow(pOverrho / sv, 1. / (g - 2.)); /* quirk: gamma-2 (rhs.c:1036) */
        RW(n) = RO(n) * Vn;
        pp = pOverrho * RO(n);
        RE(n) = pp / (g - 1.) + 0.5 * (RU(n) * RU(n) + RV(n) * RV(n) + RW(n) * RW(n)) * RO(n);
      } else if (bc[5] == 51) {
        RO(n) = 0.5; RU(n) = 0.; RV(n) = 0.; RW(n) = 0.; RE(n) = 1.4275;
      } else if (bc[5] == 10) {
        RO(n) = 1.; RU(n) = 0.; RV(n) = 0.; RW(n) = 1.; RE(n) = 1 / 0.4 + 0.5;
      } else if (bc[5] == 8) { /* subsonic non-reflecting outflow (rhs.c:1056-1086) */
        double L[5], Lambda[5], d[5], a_sound, AA;
        a_sound = sqrt(g * lp[m1] / lq[0][m1]);
        AA = RW(m1) / RO(m1);
        Lambda[0] = AA - a_sound;
        Lambda[1] = AA; Lambda[2] = AA; Lambda[3] = AA;
        Lambda[4] = AA + a_sound;
        L[0] = 0;
        L[1] = Lambda[1] * aj[m1] * zet[2][m1] * (a_sound * a_sound * (lq[0][m1] - lq[0][m2]) - (lp[n] - lp[m1]));
        L[2] = Lambda[2] * aj[m1] * zet[2][m1] * (lq[1][m1] / RO(m1) - lq[1][m2] / RO(m1)); /* TwoD 0 */
        L[3] = Lambda[3] * aj[m1] * zet[2][m1] * (lq[2][m1] / RO(m1) - lq[2][m2] / RO(m2));
        L[4] = Lambda[4] * aj[m1] * zet[2][m1] *
               ((lp[m1] - lp[m2]) + RO(m1) * a_sound * (lq[3][m1] / RO(m1) - lq[3][m2] / RO(m2)));
        d[0] = 1. / (a_sound * a_sound) * (L[1] + 0.5 * (L[4] + L[0]));
        d[1] = 0.5 * (L[0] + L[4]);
        d[2] = 0.5 / (RO(m1) * a_sound) * (L[4] - L[0]);
        d[3] = L[2];
        d[4] = L[3];
        RO(n) = qold[0][n] - c->dt * alfa * d[0];
        RE(n) = qold[4][n] - c->dt * alfa *
                                 (0.5 * d[0] * (lq[3][m1] / RO(m1) * lq[3][m1] / RO(m1)) + d[1] / (g - 1.) +
                                  lq[3][m1] * d[2]);
        RW(n) = qold[3][n] - c->dt * alfa * (lq[3][m1] / RO(m1) * d[0] + RO(m1) * d[2]);
      }
    }
#undef RO
#undef RU
#undef RV
#undef RW
#undef RE
  /* periodic copies (rhs.c:1107-1227), of Q and P alike, from lQ and the
   * local pressure as the face codes left it */
#define PCOPY(n, src)                                           \
  do {                                                          \
    for (int a = 0; a < 5; a++) q[a][n] = lq[a][src];           \
    if (p) p[n] = lp[src];                                      \
  } while (0)
  if (bc[0] == 7 || bc[1] == 7) {
    for (int k = 1; k < mz; k++)
      for (int j = 1; j < my; j++) {
        ptrdiff_t n = IX(&G, 0, j, k);
        PCOPY(n, n - 2 * si);
        n = IX(&G, mx - 1, j, k);
        PCOPY(n, n + 2 * si);
      }
  }
  if (bc[2] == 7 || bc[3] == 7) {
    for (int k = 1; k < mz; k++)
      for (int i = 0; i < mx; i++) {
        ptrdiff_t n = IX(&G, i, 0, k);
        PCOPY(n, n - 2 * sj);
      }
    for (int k = 1; k < mz - 1; k++)
      for (int i = 0; i < mx; i++) {
        ptrdiff_t n = IX(&G, i, my - 1, k);
        PCOPY(n, n + 2 * sj);
      }
  }
  if (bc[4] == 7 || bc[5] == 7) {
    for (int j = 0; j < my; j++)
      for (int i = 0; i < mx; i++) {
        ptrdiff_t n = IX(&G, i, j, 0);
        PCOPY(n, n - 2 * sk);
        n = IX(&G, i, j, mz - 1);
        PCOPY(n, n + 2 * sk);
      }
  }
#undef PCOPY
  free(lp);
  for (int a = 0; a < 5; a++) cbo_fill_ghosts(c, q[a]);
  if (p) cbo_fill_ghosts(c, p);
  return 0;
}

int cbo_formbcs(const cbo_config *c, double alfa, const double *const lq[5], const double *const qold[5],
                const double *const eta[3], const double *const zet[3], const double *aj, const double *nvert,
                double *const q[5]) {
  return formbcs_impl(c, c->ti0, alfa, lq, NULL, qold, eta, zet, aj, nvert, q, NULL);
}

int cbo_formbcs_lp(const cbo_config *c, double alfa, const double *const lq[5], const double *lp,
                   const double *const qold[5], const double *const eta[3], const double *const zet[3],
                   const double *aj, const double *nvert, double *const q[5], double *p) {
  return formbcs_impl(c, c->ti0, alfa, lq, lp, qold, eta, zet, aj, nvert, q, p);
}

/* ------------------------------------------------------------------------ */
/* Time steps  (main.c:900-974 -> Flow_Solver solvers.c:13-64 -> RungeKutta)  */
/* ------------------------------------------------------------------------ */
int cbo_steps(const cbo_config *c, int nsteps, double *const q[5], double *const qold[5],
              double *const quc[5], int *have_uc, double *nut, const double *const csi[3],
              const double *const eta[3], const double *const zet[3], const double *aj,
              const double *nvert) {
  geom G = mkgeom(c);
  int ns = cbo_nstages(c);
  double *buf = (double *)calloc(G.n * 15, sizeof(double));
  double *rhs[5], *qn[5], *sig[3], *pbuf = buf + G.n * 13, *csbuf = buf + G.n * 14;
  for (int a = 0; a < 5; a++) { rhs[a] = buf + G.n * a; qn[a] = buf + G.n * (5 + a); }
  for (int a = 0; a < 3; a++) sig[a] = buf + G.n * (10 + a);
  if (c->les && !c->calc_sigma) cbo_sigma(c, sig);
  int err = 0;
  for (int step = 0; step < nsteps && !err; step++) {
    if (cbo_les_dynamic(c) && !c->inviscid) { /* Compute_Smagorinsky_Constant_1 (dynamic), then the eddy viscosity */
      const double *const *qu = *have_uc ? (const double *const *)quc : NULL;
      cbo_eos(c, (const double *const *)q, pbuf);
      cbo_dynamic_smagorinsky(c, (const double *const *)q, qu, pbuf, csi, eta, zet, aj, nvert, csbuf);
      cbo_eddy_viscosity_dyn(c, (const double *const *)q, qu, csi, eta, zet, aj, nvert, csbuf, nut);
    } else if (c->les && c->les != 10 && !c->inviscid) /* solvers.c:28: no model at all with -les 10 */
      cbo_eddy_viscosity(c, *have_uc ? (const double *const *)quc : NULL, csi, eta, zet, aj, nvert, nut);
    for (int s = 0; s < ns && !err; s++) {
      if (c->les && c->calc_sigma && s == 0) cbo_sigma_sensor(c, (const double *const *)q, sig); /* istage 0 */
      err = cbo_rhs(c, (const double *const *)q, csi, eta, zet, aj, nvert, nut, (const double *const *)sig, rhs);
      if (err) break;
      if (!c->inviscid) { /* CalcUCat inside formRHS keeps this stage's input */
        for (int a = 0; a < 5; a++) memcpy(quc[a], q[a], G.n * sizeof(double));
        *have_uc = 1;
      }
      cbo_rk_combine(c, s, (const double *const *)qold, (const double *const *)q, (const double *const *)rhs, qn);
      {
        double al[3] = {1., 1 / 4., 2 / 3.};
        if (c->fluxorder < 3) al[1] = 1 / 2.;
        err = formbcs_impl(c, c->ti0 + step, al[s], (const double *const *)q, NULL, (const double *const *)qold, eta, zet,
                           aj, nvert, qn, NULL);
      }
      for (int a = 0; a < 5; a++) memcpy(q[a], qn[a], G.n * sizeof(double));
    }
    for (int a = 0; a < 5; a++) memcpy(qold[a], q[a], G.n * sizeof(double));
  }
  free(buf);
  return err;
}

/* ------------------------------------------------------------------------ */
/* Immersed-boundary interpolation (ibm_interpolation_advanced,              */
/* ibm_iso.c:2572-2880) with the wall models noslip / freeslip                */
/* (wallfunction.c:12-48)                                                     */
/* ------------------------------------------------------------------------ */
#define IBM_SWEEPS 5 /* itr_tmp, ibm_iso.c:2616 */

/* Surface velocity at the interception point: the element's three vertex
 * values weighted by cs1..cs3 (ibm_iso.c:2680-2690). */
static void ibm_surface_u(const cbo_ibm_surface *s, const double *u, int cell, const cbo_ibm_info *b, double U[3]) {
  const int a = s->nv1[cell], m = s->nv2[cell], z = s->nv3[cell];
  for (int d = 0; d < 3; d++) U[d] = u[3 * a + d] * b->cs1 + u[3 * m + d] * b->cs2 + u[3 * z + d] * b->cs3;
}

/* The hydset log law of the wall (wall_function_loglaw with
 * find_utau_hydset, wallfunction.c:49-100, 376-420), the model of
 * -wallfunction 2.  kappa = 0.41, B = 5.5 (wallfunction.c:10); ks is the
 * roughness (1e-16 from ibm_interpolation_advanced, ibm_iso.c:2715).  The
 * reference's operation order throughout; u_tau by Newton's method with a
 * central-difference derivative, at most 30 iterations. */
static const double WF_KAPPA = 0.41, WF_B = 5.5;

static double wf_E(double utau, double ks, double nu) { /* E_coeff, wallfunction.c:49-56 */
  double kplus = utau * ks / nu, dB;
  if (kplus <= 2.25) dB = 0.0;
  else if (kplus > 2.25 && kplus < 90.) dB = (WF_B - 8.5 + 1. / WF_KAPPA * log(kplus)) * sin(0.4258 * (log(kplus) - 0.811));
  else dB = WF_B - 8.5 + 1. / WF_KAPPA * log(kplus);
  return exp(WF_KAPPA * (WF_B - dB));
}

static double wf_u(double nu, double y, double utau, double ks) { /* u_hydset_roughness, wallfunction.c:58-67 */
  const double yplus = utau * y / nu;
  if (yplus <= 11.53) return utau * yplus;
  if (yplus <= 300) return utau / WF_KAPPA * log(wf_E(utau, ks, nu) * yplus);
  return -1.;
}

static double wf_f(double nu, double u, double y, double utau0, double ks) { /* f_hydset, wallfunction.c:69-76 */
  const double yplus = utau0 * y / nu;
  if (yplus <= 11.53) return utau0 * yplus - u;
  return utau0 * (1. / WF_KAPPA * log(wf_E(utau0, ks, nu) * yplus)) - u;
}

static double wf_find_utau(double nu, double u, double y, double guess, double ks) { /* wallfunction.c:78-100 */
  const double eps = 1.e-7;
  double utau = guess, utau0 = guess;
  for (int ii = 0; ii < 30; ii++) {
    const double df = (wf_f(nu, u, y, utau0 + eps, ks) - wf_f(nu, u, y, utau0 - eps, ks)) / (2. * eps);
    utau = utau0 - wf_f(nu, u, y, utau0, ks) / df;
    if (fabs(utau - utau0) < 1.e-7) break;
    utau0 = utau;
  }
  return utau;
}

/* Ub of the log-law wall (wall_function_loglaw, wallfunction.c:376-420):
 * the tangential part of the donor velocity scaled to the modelled
 * magnitude at sb, the normal part linear in the distance. */
static void wf_loglaw(double nu, double ks, double sc, double sb, const double Ua[3], const double Uc[3], double Ub[3],
                      double *ustar, double nx, double ny, double nz) {
  const double u_c = Uc[0] - Ua[0], v_c = Uc[1] - Ua[1], w_c = Uc[2] - Ua[2];
  const double un = u_c * nx + v_c * ny + w_c * nz;
  double ut = u_c - un * nx, vt = v_c - un * ny, wt = w_c - un * nz;
  const double ut_mag = sqrt(ut * ut + vt * vt + wt * wt);
  *ustar = wf_find_utau(nu, ut_mag, sc, 0.001, ks);
  double model = wf_u(nu, sb, *ustar, ks);
  if (model < 0.) model = ut_mag;
  if (ut_mag > 1.e-10) {
    ut *= model / ut_mag;
    vt *= model / ut_mag;
    wt *= model / ut_mag;
  } else {
    ut = vt = wt = 0;
  }
  Ub[0] = ut + (sb / sc * un) * nx;
  Ub[1] = vt + (sb / sc * un) * ny;
  Ub[2] = wt + (sb / sc * un) * nz;
  Ub[0] += Ua[0];
  Ub[1] += Ua[1];
  Ub[2] += Ua[2];
}

int cbo_ibm_interpolate(const cbo_config *c, const cbo_ibm_surface *s, int n, const cbo_ibm_info *list,
                        const double *const coor[3], double *const q[5], double *p, const double *const qold[5],
                        int add_dundt, int twoD, int wallfunction, double *ustar) {
  /* -wallfunction 1 reads a table that pre_integrate builds in a stack array
   * of its own frame (wallfunction.c:113-145): undefined once it returns */
  if (wallfunction == 1) return 5; /* not restated */
  geom G = mkgeom(c);
  double *buf = (double *)malloc(G.n * 7 * sizeof(double));
  double *lq[5], *lp = buf + G.n * 5, *rho_old = buf + G.n * 6;
  for (int a = 0; a < 5; a++) lq[a] = buf + G.n * a;
  /* Qold's density for the characteristic wall: the step's start state, or
   * the state as given */
  memcpy(rho_old, qold ? qold[0] : q[0], G.n * sizeof(double));
  const double gm2 = c->gamma * c->ma * c->ma;
  /* -isothermal 2 (ibm_iso.c:2744-2786): one scalar Pa, the pressure of the
   * previous entry walked (the entry's own at sweep 0), links the entries */
  double Pa = 0.;
  const int slip = c->inviscid || wallfunction == 3; /* ibm_iso.c:2721 */
  for (int sweep = 0; sweep < IBM_SWEEPS; sweep++) {
    /* the sweep reads the local vectors lQ / lP and writes the global Q / P */
    for (int a = 0; a < 5; a++) memcpy(lq[a], q[a], G.n * sizeof(double));
    memcpy(lp, p, G.n * sizeof(double));
    for (int e = 0; e < n; e++) {
      const cbo_ibm_info *b = &list[e];
      const ptrdiff_t o = IX(&G, b->ni, b->nj, b->nk);
      const ptrdiff_t d1 = IX(&G, b->i1, b->j1, b->k1), d2 = IX(&G, b->i2, b->j2, b->k2),
                      d3 = IX(&G, b->i3, b->j3, b->k3);
      const double sb = b->d_s, sc = sb + b->d_i;
      const double sk1 = b->cr1, sk2 = b->cr2, sk3 = b->cr3;
      /* direction from the interception point to the node (ibm_iso.c:2662-2681) */
      double nfx = twoD == 1 ? 0. : coor[0][o] - b->pmin[0];
      double nfy = twoD == 2 ? 0. : coor[1][o] - b->pmin[1];
      double nfz = twoD == 3 ? 0. : coor[2][o] - b->pmin[2];
      const double dr = sqrt(nfx * nfx + nfy * nfy + nfz * nfz);
      if (dr < 0.000000001) {
        if (b->cell >= 0) { nfx = s->nf_x[b->cell]; nfy = s->nf_y[b->cell]; nfz = s->nf_z[b->cell]; }
        else { nfx = 0.; nfy = 0.; nfz = 0.; }
      } else {
        nfx = nfx / dr; nfy = nfy / dr; nfz = nfz / dr;
      }
      double Ua[3] = {0., 0., 0.}, Ua_n = 0., Ua_nold = 0.;
      if (b->cell >= 0) {
        ibm_surface_u(s, s->uold, b->cell, b, Ua);
        Ua_nold = Ua[0] * nfx + Ua[1] * nfy + Ua[2] * nfz;
        ibm_surface_u(s, s->u, b->cell, b, Ua);
        Ua_n = Ua[0] * nfx + Ua[1] * nfy + Ua[2] * nfz;
      }
      /* velocity at the donor point (ibm_iso.c:2704-2706) */
      double Uc[3];
      for (int d = 0; d < 3; d++)
        Uc[d] = lq[1 + d][d1] / lq[0][d1] * sk1 + lq[1 + d][d2] / lq[0][d2] * sk2 + lq[1 + d][d3] / lq[0][d3] * sk3;
      double Ub[3];
      if (wallfunction == 2) { /* ibm_iso.c:2714-2719, 1/user->ren as the reference */
        double us;
        wf_loglaw(1. / c->ren, 1.e-16, sc, sb, Ua, Uc, Ub, &us, nfx, nfy, nfz);
        if (ustar) ustar[e] = us;
      } else if (slip) { /* freeslip: normal part linear in the distance, tangential part of the donor */
        const double Uan = Ua[0] * nfx + Ua[1] * nfy + Ua[2] * nfz;
        const double Ucn = Uc[0] * nfx + Uc[1] * nfy + Uc[2] * nfz;
        const double Ubn = Uan + (Ucn - Uan) * sb / sc;
        const double nv[3] = {nfx, nfy, nfz};
        for (int d = 0; d < 3; d++) Ub[d] = (Uc[d] - Ucn * nv[d]) + Ubn * nv[d];
      } else { /* noslip: linear between the wall velocity and the donor */
        for (int d = 0; d < 3; d++) Ub[d] = sb / sc * (Uc[d] - Ua[d]) + Ua[d];
      }
      double pb = lp[d1] * sk1 + lp[d2] * sk2 + lp[d3] * sk3;
      if (twoD == 1) Ub[0] = 0.;
      if (twoD == 2) Ub[1] = 0.;
      if (twoD == 3) Ub[2] = 0.;
      double rho;
      if (c->isothermal == 2) {
        /* the no-slip isothermal wall of Poinsot & Lele (J. Comput. Phys. 101,
         * 1992) through the incoming characteristic u_n - a, with a^2 = Twall
         * / Ma^2 and the wall temperature Tb interpolated like the velocity */
        const double rhoc = lq[0][d1] * sk1 + lq[0][d2] * sk2 + lq[0][d3] * sk3;
        double Tc = pb / rhoc * gm2;
        if (Tc < 0.) Tc = 0.;
        const double Tb = (Tc - c->twall) * sb / sc + c->twall;
        const double a_sound = sqrt(c->twall / (c->ma * c->ma));
        const double Lambda1 = Ua_n - a_sound;
        if (sweep == 0) Pa = pb;
        const double L1 = Lambda1 / sc *
                          ((pb - Pa) - rhoc * a_sound * ((Uc[0] - Ua[0]) * nfx + (Uc[1] - Ua[1]) * nfy +
                                                         (Uc[2] - Ua[2]) * nfz));
        rho = rho_old[o] - c->dt * L1 / a_sound / a_sound;
        pb = rho * Tb / gm2;
        Pa = pb;
      } else if (c->isothermal == 1) {
        rho = pb * gm2 / 1.0; /* wall temperature Tb = 1 (ibm_iso.c:2795-2803) */
      } else {
        rho = lq[0][d1] * sk1 + lq[0][d2] * sk2 + lq[0][d3] * sk3; /* d rho / dn = 0 */
      }
      if (add_dundt) pb += rho * (Ua_n - Ua_nold) / c->dt * (sc - sb);
      const double ru = rho * Ub[0], rv = rho * Ub[1], rw = rho * Ub[2];
      q[0][o] = rho; q[1][o] = ru; q[2][o] = rv; q[3][o] = rw;
      q[4][o] = pb / (c->gamma - 1) + 0.5 * (ru * ru + rv * rv + rw * rw) / rho;
      p[o] = pb;
    }
    /* DMGlobalToLocal of Q and P after each sweep */
    for (int a = 0; a < 5; a++) cbo_fill_ghosts(c, q[a]);
    cbo_fill_ghosts(c, p);
  }
  free(buf);
  return 0;
}

/* Time steps with immersed bodies (RungeKutta with -imm, solvers.c:245-288):
 * the stages as in cbo_steps, EqOfState, the interpolation of each body
 * (Add_dUndt = 1), then FormBCS(user, 0), which copies Q and P across the
 * periodic boundaries and ends with their ghost wrap.  No EqOfState follows,
 * so the next step's first stage reads the pressure lp carried from here
 * (*lp_valid set) instead of the EqOfState of its input. */
int cbo_steps_ibm(const cbo_config *c, int nsteps, double *const q[5], double *const qold[5],
                  double *const quc[5], int *have_uc, double *nut, const double *const csi[3],
                  const double *const eta[3], const double *const zet[3], const double *aj,
                  const double *nvert, int nbodies, const cbo_ibm_surface *surf, const int *nlist,
                  const cbo_ibm_info *const *lists, const double *const coor[3], double *lp, int *lp_valid,
                  int twoD, int wallfunction) {
  geom G = mkgeom(c);
  int ns = cbo_nstages(c);
  double *buf = (double *)calloc(G.n * 20, sizeof(double));
  double *rhs[5], *qn[5], *sig[3], *lq[5], *lpc = buf + G.n * 18, *csbuf = buf + G.n * 19;
  for (int a = 0; a < 5; a++) { rhs[a] = buf + G.n * a; qn[a] = buf + G.n * (5 + a); lq[a] = buf + G.n * (13 + a); }
  for (int a = 0; a < 3; a++) sig[a] = buf + G.n * (10 + a);
  if (c->les) cbo_sigma(c, sig);
  double al[3] = {1., 1 / 4., 2 / 3.};
  if (c->fluxorder < 3) al[1] = 1 / 2.;
  int err = 0;
  for (int step = 0; step < nsteps && !err; step++) {
    if (cbo_les_dynamic(c) && !c->inviscid) { /* the dynamic model reads lP only for beta, which feeds nothing */
      const double *const *qu = *have_uc ? (const double *const *)quc : NULL;
      cbo_dynamic_smagorinsky(c, (const double *const *)q, qu, lp, csi, eta, zet, aj, nvert, csbuf);
      cbo_eddy_viscosity_dyn(c, (const double *const *)q, qu, csi, eta, zet, aj, nvert, csbuf, nut);
    } else if (c->les && c->les != 10 && !c->inviscid) /* solvers.c:28: no model at all with -les 10 */
      cbo_eddy_viscosity(c, *have_uc ? (const double *const *)quc : NULL, csi, eta, zet, aj, nvert, nut);
    for (int s = 0; s < ns && !err; s++) {
      const double *lps = (s == 0 && *lp_valid) ? lp : NULL;
      if (c->les && c->calc_sigma && s == 0) { /* istage 0 reads lP: the carried pressure when there is one */
        if (lps) cbo_sigma_sensor_p(c, lps, sig);
        else cbo_sigma_sensor(c, (const double *const *)q, sig);
      }
      err = rhs_impl(c, (const double *const *)q, lps, csi, eta, zet, aj, nvert, nut, (const double *const *)sig,
                     rhs);
      if (err) break;
      if (!c->inviscid) {
        for (int a = 0; a < 5; a++) memcpy(quc[a], q[a], G.n * sizeof(double));
        *have_uc = 1;
      }
      cbo_rk_combine(c, s, (const double *const *)qold, (const double *const *)q, (const double *const *)rhs, qn);
      err = formbcs_impl(c, c->ti0 + step, al[s], (const double *const *)q, lps, (const double *const *)qold, eta, zet, aj, nvert, qn,
                         NULL);
      for (int a = 0; a < 5; a++) memcpy(q[a], qn[a], G.n * sizeof(double));
    }
    if (err) break;
    cbo_eos(c, (const double *const *)q, lp); /* EqOfState after the last stage (solvers.c:279) */
    for (int b = 0; b < nbodies && !err; b++)
      if (nlist[b] > 0)
        err = cbo_ibm_interpolate(c, &surf[b], nlist[b], lists[b], coor, q, lp, (const double *const *)qold, 1, twoD,
                                  wallfunction, NULL);
    if (err) break;
    for (int a = 0; a < 5; a++) memcpy(lq[a], q[a], G.n * sizeof(double));
    memcpy(lpc, lp, G.n * sizeof(double));
    err = formbcs_impl(c, c->ti0 + step, 0.0, (const double *const *)lq, lpc, (const double *const *)qold, eta, zet, aj, nvert, q,
                       lp);
    *lp_valid = 1;
    for (int a = 0; a < 5; a++) memcpy(qold[a], q[a], G.n * sizeof(double));
  }
  free(buf);
  return err;
}

/* ------------------------------------------------------------------------ */
/* Dynamic Smagorinsky  (Compute_Smagorinsky_Constant_1 with -les 2,          */
/* les.c:135-1472: the default 3-D box test filter, local averaging)          */
/* ------------------------------------------------------------------------ */
#define DYN_EPS 0.000001 /* les.c:8 */

static int interior(const geom *G, int i, int j, int k) {
  return i >= 1 && i <= G->m[0] - 2 && j >= 1 && j <= G->m[1] - 2 && k >= 1 && k <= G->m[2] - 2;
}

/* integrate_testfilter (les.c:80-132): sum w*val and w in k, j, i order */
static double itf(const double val[27], const double w[27]) {
  double vs = 0.0, ws = 0.0;
  for (int t = 0; t < 27; t++) { vs += w[t] * val[t]; ws += w[t]; }
  return vs / ws;
}

/* boundary copies from two nodes across of the periodic directions over the
 * interior ranges of the other two (les.c:287-353, 1217-1271) */
static void dyn_periodic_copies(const cbo_config *c, const geom *G, double *f) {
  const int mx = G->m[0], my = G->m[1], mz = G->m[2];
  const int *bc = c->bctype;
  if (bc[0] == 7 || bc[1] == 7)
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++) {
        f[IX(G, 0, j, k)] = f[IX(G, -2, j, k)];
        f[IX(G, mx - 1, j, k)] = f[IX(G, mx + 1, j, k)];
      }
  if (bc[2] == 7 || bc[3] == 7)
    for (int k = 1; k < mz - 1; k++)
      for (int i = 1; i < mx - 1; i++) {
        f[IX(G, i, 0, k)] = f[IX(G, i, -2, k)];
        f[IX(G, i, my - 1, k)] = f[IX(G, i, my + 1, k)];
      }
  if (bc[4] == 7 || bc[5] == 7)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        f[IX(G, i, j, 0)] = f[IX(G, i, j, -2)];
        f[IX(G, i, j, mz - 1)] = f[IX(G, i, j, mz + 1)];
      }
}

/* Velocity component a the reference's lUcat holds at node m once the first
 * loop of the dynamic model has overwritten it in place: rhoU/rho of the
 * current state q at interior nodes with nvert <= 1.1 (a node the loop has
 * reached, when `reached` restricts it), else the value CalcUCat left from
 * quc (zero before any CalcUCat). */
static double dyn_u(const geom *G, const double *const q[5], const double *const quc[5], const double *nvert, int a,
                    int i, int j, int k, int reached, int twod) {
  const ptrdiff_t m = IX(G, i, j, k);
  if (reached && interior(G, i, j, k) && nvert[m] <= 1.1) return q[1 + a][m] / q[0][m]; /* les.c:255 ignores -twoD */
  if (a == 0 && twod == 1) return 0.0; /* the last CalcUCat's x with -twoD 1 (rhs.c:1349) */
  return quc ? quc[1 + a][m] / quc[0][m] : 0.0;
}

/* Homogeneous averaging of LM and MM before the clipping (les.c:934-1115), as
 * one rank sums them: running sums in k, j, i loop order.
 *  - i and k: per j plane over the fluid interior (nvert < 0.1) nodes; every
 *    interior node of the plane gets 0.5 <LM> / (<MM> + eps);
 *  - i without k: per (k, j) line along i, written at fluid interior nodes;
 *  - i, j and k: afterwards, sum LM / sum MM over every interior node
 *    (no mask, no eps, no 0.5) on every node of the box.
 * The j- and k-only branches of the reference are commented out: those
 * filters only make LM / MM pointwise. */
static void dyn_homogeneous(const cbo_config *c, const geom *G, const double *nvert, const double *LM,
                            const double *MM, double *cs) {
  const int mx = G->m[0], my = G->m[1], mz = G->m[2];
  if (c->i_homo_filter && c->k_homo_filter) {
    double *lm = (double *)calloc((size_t)my * 2, sizeof(double)), *mm = lm + my;
    int *cnt = (int *)calloc((size_t)my, sizeof(int));
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
          const ptrdiff_t n = IX(G, i, j, k);
          if (nvert[n] < 0.1) { lm[j] += LM[n]; mm[j] += MM[n]; cnt[j]++; }
        }
    for (int j = 0; j < my; j++)
      if (cnt[j] > 0) { lm[j] /= (double)cnt[j]; mm[j] /= (double)cnt[j]; }
    for (int j = 1; j < my - 1; j++)
      for (int k = 1; k < mz - 1; k++)
        for (int i = 1; i < mx - 1; i++) cs[IX(G, i, j, k)] = 0.5 * lm[j] / (mm[j] + DYN_EPS);
    free(lm);
    free(cnt);
  }
  if (c->i_homo_filter && !c->k_homo_filter) {
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++) {
        double lm = 0.0, mm = 0.0;
        int cnt = 0;
        for (int i = 1; i < mx - 1; i++) {
          const ptrdiff_t n = IX(G, i, j, k);
          if (nvert[n] < 0.1) { lm += LM[n]; mm += MM[n]; cnt++; }
        }
        if (cnt > 0) { lm /= (double)cnt; mm /= (double)cnt; }
        for (int i = 1; i < mx - 1; i++) {
          const ptrdiff_t n = IX(G, i, j, k);
          if (nvert[n] < 0.1) cs[n] = 0.5 * lm / (mm + DYN_EPS);
        }
      }
  }
  if (c->i_homo_filter && c->j_homo_filter && c->k_homo_filter) {
    double lm = 0.0, mm = 0.0;
    for (int k = 1; k < mz - 1; k++)
      for (int j = 1; j < my - 1; j++)
        for (int i = 1; i < mx - 1; i++) {
          const ptrdiff_t n = IX(G, i, j, k);
          mm += MM[n];
          lm += LM[n];
        }
    for (int k = 0; k < mz; k++)
      for (int j = 0; j < my; j++)
        for (int i = 0; i < mx; i++) cs[IX(G, i, j, k)] = lm / mm;
  }
}

int cbo_les_dynamic(const cbo_config *c) { return c->les >= 2 && c->les != 10; }

int cbo_dynamic_smagorinsky(const cbo_config *c, const double *const q[5], const double *const quc[5],
                            const double *lp, const double *const csi[3], const double *const eta[3],
                            const double *const zet[3], const double *aj, const double *nvert, double *cs) {
  const double max_cs = c->max_cs;
  geom G = mkgeom(c);
  const int mx = G.m[0], my = G.m[1], mz = G.m[2];
  if (!cbo_les_dynamic(c)) return 5;
  /* -les 3 and the homogeneous filters take LM / MM node by node and skip
   * the final 1/aj-weighted mean (les.c:916-922, 1302) */
  const int pointwise = c->i_homo_filter || c->j_homo_filter || c->k_homo_filter || c->les == 3;
  double *buf = (double *)calloc(G.n * 13, sizeof(double));
  double *A[9], *Sabs = buf + 9 * G.n, *LM = buf + 10 * G.n, *MM = buf + 11 * G.n, *ct = buf + 12 * G.n;
  for (int a = 0; a < 9; a++) A[a] = buf + a * G.n; /* du_dx du_dy du_dz dv_dx .. dw_dz */
  /* (1) velocity gradients and |S| at interior nodes (les.c:234-284), the
   * velocity overwritten in loop order: the -1 neighbours are already new */
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const ptrdiff_t n = IX(&G, i, j, k);
        if (nvert[n] > 1.1) continue;
        double d[3][3];
        for (int a = 0; a < 3; a++) {
          d[a][0] = (dyn_u(&G, q, quc, nvert, a, i + 1, j, k, 0, c->twod) - dyn_u(&G, q, quc, nvert, a, i - 1, j, k, 1, c->twod)) * 0.5;
          d[a][2] = (dyn_u(&G, q, quc, nvert, a, i, j, k + 1, 0, c->twod) - dyn_u(&G, q, quc, nvert, a, i, j, k - 1, 1, c->twod)) * 0.5;
          d[a][1] = (dyn_u(&G, q, quc, nvert, a, i, j + 1, k, 0, c->twod) - dyn_u(&G, q, quc, nvert, a, i, j - 1, k, 1, c->twod)) * 0.5;
        }
        const double ajc = aj[n];
        const double c0 = csi[0][n], c1 = csi[1][n], c2 = csi[2][n];
        const double e0 = eta[0][n], e1 = eta[1][n], e2 = eta[2][n];
        const double z0 = zet[0][n], z1 = zet[1][n], z2 = zet[2][n];
        double g[3][3];
        for (int a = 0; a < 3; a++) {
          g[a][0] = (d[a][0] * c0 + d[a][1] * e0 + d[a][2] * z0) * ajc;
          g[a][1] = (d[a][0] * c1 + d[a][1] * e1 + d[a][2] * z1) * ajc;
          g[a][2] = (d[a][0] * c2 + d[a][1] * e2 + d[a][2] * z2) * ajc;
        }
        const double Sdd = 2. / 3. * (g[0][0] + g[1][1] + g[2][2]);
        const double Sxx = 0.5 * (g[0][0] + g[0][0]) - Sdd, Sxy = 0.5 * (g[0][1] + g[1][0]), Sxz = 0.5 * (g[0][2] + g[2][0]);
        const double Syx = Sxy, Syy = 0.5 * (g[1][1] + g[1][1]) - Sdd, Syz = 0.5 * (g[1][2] + g[2][1]);
        const double Szx = Sxz, Szy = Syz, Szz = 0.5 * (g[2][2] + g[2][2]) - Sdd;
        Sabs[n] = sqrt(2.0 * (Sxx * Sxx + Sxy * Sxy + Sxz * Sxz + Syx * Syx + Syy * Syy + Syz * Syz + Szx * Szx +
                              Szy * Szy + Szz * Szz));
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) A[3 * a + b][n] = g[a][b];
      }
  /* DMLocalToLocal of the gradients and |S|, then the gradients' periodic copies */
  for (int a = 0; a < 9; a++) cbo_fill_ghosts(c, A[a]);
  cbo_fill_ghosts(c, Sabs);
  for (int a = 0; a < 9; a++) dyn_periodic_copies(c, &G, A[a]);
  /* (2) Germano identity with the 3x3x3 box test filter (les.c:442-792) */
  double w[27];
  for (int R = 0; R < 3; R++)
    for (int Q = 0; Q < 3; Q++)
      for (int P = 0; P < 3; P++)
        w[(R * 3 + Q) * 3 + P] = 1. / (fabs(R - 1.0) + 1) * 1. / (fabs(Q - 1.0) + 1) * 1. / (fabs(P - 1.0) + 1);
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const ptrdiff_t n = IX(&G, i, j, k);
        if (nvert[n] > 1.1) { LM[n] = MM[n] = 0; continue; }
        double u[27], v[27], ww[27], rho[27], ru[27], rv[27], rw[27], ruu[27], ruv[27], ruw[27], rvv[27], rvw[27],
            rww[27], S[9][27], SS[9][27], pu[27], pv[27], pw[27], pp[27];
        for (int R = 0; R < 3; R++)
          for (int Q = 0; Q < 3; Q++)
            for (int P = 0; P < 3; P++) {
              const int t = (R * 3 + Q) * 3 + P;
              const int II = i + P - 1, JJ = j + Q - 1, KK = k + R - 1;
              const ptrdiff_t m = IX(&G, II, JJ, KK);
              u[t] = dyn_u(&G, q, quc, nvert, 0, II, JJ, KK, 1, c->twod);
              v[t] = dyn_u(&G, q, quc, nvert, 1, II, JJ, KK, 1, c->twod);
              ww[t] = dyn_u(&G, q, quc, nvert, 2, II, JJ, KK, 1, c->twod);
              ru[t] = q[1][m]; rv[t] = q[2][m]; rw[t] = q[3][m]; rho[t] = q[0][m];
              ruu[t] = ru[t] * u[t]; ruv[t] = ru[t] * v[t]; ruw[t] = ru[t] * ww[t];
              rvv[t] = rv[t] * v[t]; rvw[t] = rv[t] * ww[t]; rww[t] = rw[t] * ww[t];
              const double du_dx = A[0][m], du_dy = A[1][m], du_dz = A[2][m];
              const double dv_dx = A[3][m], dv_dy = A[4][m], dv_dz = A[5][m];
              const double dw_dx = A[6][m], dw_dy = A[7][m], dw_dz = A[8][m];
              const double Sxx = 0.5 * (du_dx + du_dx), Sxy = 0.5 * (du_dy + dv_dx), Sxz = 0.5 * (du_dz + dw_dx);
              const double Syy = 0.5 * (dv_dy + dv_dy), Syz = 0.5 * (dv_dz + dw_dy);
              const double Szz = 0.5 * (dw_dz + dw_dz);
              const double s9[9] = {Sxx, Sxy, Sxz, Sxy, Syy, Syz, Sxz, Syz, Szz};
              for (int a = 0; a < 9; a++) {
                S[a][t] = s9[a];
                SS[a][t] = s9[a] * Sabs[m] * rho[t];
              }
              pu[t] = u[t] * lp[m]; pv[t] = v[t] * lp[m]; pw[t] = ww[t] * lp[m]; pp[t] = lp[m];
            }
        (void)pu; (void)pv; (void)pw; (void)pp; /* beta (les.c:578-581) feeds nothing downstream */
        const double filter = pow(1. / aj[n], 1. / 3.);
        const double test_filter = c->testfilter_ik ? pow(5.0, 1. / 3.) * filter : 2.0 * filter; /* les.c:598-601 */
        const double _rho = itf(rho, w), _rhou = itf(ru, w), _rhov = itf(rv, w), _rhow = itf(rw, w);
        double Lij[3][3];
        Lij[0][0] = itf(ruu, w) - _rhou * _rhou / _rho;
        Lij[0][1] = itf(ruv, w) - _rhou * _rhov / _rho;
        Lij[0][2] = itf(ruw, w) - _rhou * _rhow / _rho;
        Lij[1][0] = itf(ruv, w) - _rhov * _rhou / _rho;
        Lij[1][1] = itf(rvv, w) - _rhov * _rhov / _rho;
        Lij[1][2] = itf(rvw, w) - _rhov * _rhow / _rho;
        Lij[2][0] = itf(ruw, w) - _rhow * _rhou / _rho;
        Lij[2][1] = itf(rvw, w) - _rhow * _rhov / _rho;
        Lij[2][2] = itf(rww, w) - _rhow * _rhow / _rho;
        double Sxyz[3][3], Sh[3][3], SSh[3][3];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) {
            Sxyz[a][b] = S[3 * a + b][13];
            Sh[a][b] = itf(S[3 * a + b], w);
            SSh[a][b] = itf(SS[3 * a + b], w);
          }
        double S_hat = 0;
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) S_hat += pow(Sh[a][b], 2.);
        S_hat = sqrt(2 * S_hat);
        double L_cat = 0.0, M_cat = 0.0;
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) {
            M_cat += -2.0 * _rho * pow(test_filter, 2.) * S_hat * (Sh[a][b] * Sxyz[a][b] - 0.33 * Sh[a][a] * Sxyz[b][b]) +
                     2.0 * pow(filter, 2.) * (SSh[a][b] * Sxyz[a][b] - 0.33 * SSh[a][a] * Sxyz[b][b]);
            L_cat += Lij[a][b] * Sxyz[a][b] - 0.33 * Sxyz[a][a] * Lij[b][b];
          }
        LM[n] = L_cat;
        MM[n] = M_cat;
      }
  cbo_fill_ghosts(c, LM);
  cbo_fill_ghosts(c, MM);
  /* (3) Cs from the 27-node mean of LM and MM (les.c:905-925) */
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const ptrdiff_t n = IX(&G, i, j, k);
        if (nvert[n] > 1.1) { cs[n] = 0; continue; }
        double lm = 0.0, mm = 0.0; /* integrate_t (les.c:66-78) */
        if (pointwise) {
          lm = LM[n];
          mm = MM[n];
        } else {
          for (int R = 0; R < 3; R++)
            for (int Q = 0; Q < 3; Q++)
              for (int P = 0; P < 3; P++) {
                const ptrdiff_t m = IX(&G, i + P - 1, j + Q - 1, k + R - 1);
                lm += LM[m] / 27.0;
                mm += MM[m] / 27.0;
              }
        }
        const double C = lm / (mm + DYN_EPS);
        cs[n] = (C < 0.0001) ? 0.0001 : C;
      }
  dyn_homogeneous(c, &G, nvert, LM, MM, cs);
  /* (4) clipping on every owned node (les.c:1124-1137; its face tests compare
   * !bctype with 7 and never hold) */
  for (int k = 0; k < mz; k++)
    for (int j = 0; j < my; j++)
      for (int i = 0; i < mx; i++) {
        const ptrdiff_t n = IX(&G, i, j, k);
        if (nvert[n] > 1.1 && nvert[n] < 7.) { cs[n] = 0.0; continue; }
        if (nvert[n] > 0.1 && nvert[n] < 1.1) cs[n] = (0.01 < cs[n]) ? cs[n] : 0.01; /* PetscMax(0.01, Cs) */
        const double t = (cs[n] < 0.000) ? 0.000 : cs[n];
        cs[n] = (t < max_cs) ? t : max_cs;
      }
  /* (5) lCS with its periodic copies, then the 1/aj-weighted mean over the
   * 27 nodes around fluid interior nodes (les.c:1207-1333) */
  if (pointwise) {
    free(buf);
    return 0;
  }
  memcpy(ct, cs, G.n * sizeof(double));
  cbo_fill_ghosts(c, ct);
  dyn_periodic_copies(c, &G, ct);
  for (int k = 1; k < mz - 1; k++)
    for (int j = 1; j < my - 1; j++)
      for (int i = 1; i < mx - 1; i++) {
        const ptrdiff_t n = IX(&G, i, j, k);
        if (!(nvert[n] < 0.1)) continue;
        double wt[27], C[27];
        for (int R = 0; R < 3; R++)
          for (int Q = 0; Q < 3; Q++)
            for (int P = 0; P < 3; P++) {
              const int t = (R * 3 + Q) * 3 + P;
              const ptrdiff_t m = IX(&G, i + P - 1, j + Q - 1, k + R - 1);
              wt[t] = 1. / aj[m];
              C[t] = ct[m];
            }
        cs[n] = itf(C, wt);
      }
  free(buf);
  return 0;
}

/* Compute_eddy_viscosity_LES (les.c:1523-1567) after the dynamic model: Cs
 * per node, and the velocity the model left in lUcat (see dyn_u). */
void cbo_eddy_viscosity_dyn(const cbo_config *c, const double *const q[5], const double *const quc[5],
                            const double *const csi[3], const double *const eta[3], const double *const zet[3],
                            const double *aj, const double *nvert, const double *cs, double *nut) {
  geom G = mkgeom(c);
  for (int k = 1; k < G.m[2] - 1; k++)
    for (int j = 1; j < G.m[1] - 1; j++)
      for (int i = 1; i < G.m[0] - 1; i++) {
        const ptrdiff_t n = IX(&G, i, j, k);
        if (nvert[n] > 0.1) { nut[n] = 0; continue; }
        double d[3][3];
        for (int a = 0; a < 3; a++) {
          d[a][0] = (dyn_u(&G, q, quc, nvert, a, i + 1, j, k, 1, c->twod) - dyn_u(&G, q, quc, nvert, a, i - 1, j, k, 1, c->twod)) * 0.5;
          d[a][1] = (dyn_u(&G, q, quc, nvert, a, i, j + 1, k, 1, c->twod) - dyn_u(&G, q, quc, nvert, a, i, j - 1, k, 1, c->twod)) * 0.5;
          d[a][2] = (dyn_u(&G, q, quc, nvert, a, i, j, k + 1, 1, c->twod) - dyn_u(&G, q, quc, nvert, a, i, j, k - 1, 1, c->twod)) * 0.5;
        }
        const double ajc = aj[n];
        const double c0 = csi[0][n], c1 = csi[1][n], c2 = csi[2][n];
        const double e0 = eta[0][n], e1 = eta[1][n], e2 = eta[2][n];
        const double z0 = zet[0][n], z1 = zet[1][n], z2 = zet[2][n];
        double g[3][3];
        for (int a = 0; a < 3; a++) {
          g[a][0] = (d[a][0] * c0 + d[a][1] * e0 + d[a][2] * z0) * ajc;
          g[a][1] = (d[a][0] * c1 + d[a][1] * e1 + d[a][2] * z1) * ajc;
          g[a][2] = (d[a][0] * c2 + d[a][1] * e2 + d[a][2] * z2) * ajc;
        }
        const double Sdd = 2. / 3. * (g[0][0] + g[1][1] + g[2][2]);
        const double Sxx = 0.5 * (g[0][0] + g[0][0]) - Sdd, Sxy = 0.5 * (g[0][1] + g[1][0]), Sxz = 0.5 * (g[0][2] + g[2][0]);
        const double Syx = Sxy, Syy = 0.5 * (g[1][1] + g[1][1]) - Sdd, Syz = 0.5 * (g[1][2] + g[2][1]);
        const double Szx = Sxz, Szy = Syz, Szz = 0.5 * (g[2][2] + g[2][2]) - Sdd;
        const double Sabs = sqrt(2.0 * (Sxx * Sxx + Sxy * Sxy + Sxz * Sxz + Syx * Syx + Syy * Syy + Syz * Syz +
                                        Szx * Szx + Szy * Szy + Szz * Szz));
        const double filter = pow(1. / aj[n], 1. / 3.);
        nut[n] = cs[n] * pow(filter, 2.0) * Sabs;
      }
  cbo_fill_ghosts(c, nut);
}
