// Auxiliary kernels: periodic boundary/ghost fill (FormBCS + DMGlobalToLocal),
// eddy viscosity (Compute_eddy_viscosity_LES), device metrics (FormMetrics),
// AoS <-> padded SoA packing and the EOS for downloads.  All are HBM-bound
// elementwise/stencil sweeps; grids are sized in multiples of the SM count
// by the host and every kernel uses a grid-stride loop.
#pragma once
#include "cb_common.cuh"

namespace cb {

__device__ __forceinline__ int wrapi(int x, int m) { return x < 0 ? x + m : (x >= m ? x - m : x); }

// Final value source of a non-interior node after FormBCS (fully periodic):
// boundary nodes take the stale stage input at the periodic image two nodes
// across (rhs.c:1107-1227; later copies win: k faces, then j, then i), the
// ghost layers then wrap onto the updated global vector (DMGlobalToLocal).
// Returns true and sets (si,sj,sk,from_in) for a boundary/ghost node.
__device__ __forceinline__ void bc_source(const DevCfg &c, int i, int j, int k, int &si, int &sj, int &sk, bool &from_in) {
  // ghost -> owned image
  int oi = wrapi(i, c.mx), oj = wrapi(j, c.my), ok = wrapi(k, c.mz);
  si = oi; sj = oj; sk = ok; from_in = false;
  const bool bnd = oi == 0 || oi == c.mx - 1 || oj == 0 || oj == c.my - 1 || ok == 0 || ok == c.mz - 1;
  if (!bnd) return;  // image is interior: value of the stage output
  from_in = true;
  if (ok == 0) sk = ok - 2;
  else if (ok == c.mz - 1) sk = ok + 2;
  else if (oj == 0) sj = oj - 2;
  else if (oj == c.my - 1) sj = oj + 2;
  else if (oi == 0) si = oi - 2;
  else si = oi + 2;  // oi == mx-1
}

// The non-interior nodes of the padded box (three layers on each side: two
// ghost layers and the boundary layer), enumerated without the interior: six
// full planes, then per middle plane six full rows and six side nodes per
// middle row.
__host__ __device__ __forceinline__ long long shell_count(const DevCfg &c) {
  const long long NX = c.mx + 4, NY = c.my + 4;
  return 6 * NX * NY + (long long)(c.mz - 2) * (6 * NX + 6 * (c.my - 2));
}
// 32-bit index arithmetic (a shell count below 2^31 is checked on the host):
// 64-bit division costs far more than the copy it addresses.
__device__ __forceinline__ void shell_node(const DevCfg &c, long long t64, int &i, int &j, int &k) {
  const unsigned t = (unsigned)t64;
  const unsigned NX = c.mx + 4, NY = c.my + 4, NZ = c.mz + 4, A = NX * NY, Pm = 6 * NX + 6 * (c.my - 2);
  unsigned I, J, K;
  if (t < 6 * A) {
    const unsigned p = t / A, r = t - p * A;
    K = p < 3 ? p : NZ - 6 + p;
    J = r / NX;
    I = r - J * NX;
  } else {
    const unsigned t2 = t - 6 * A;
    K = 3 + t2 / Pm;
    const unsigned r = t2 - (K - 3) * Pm;
    if (r < 6 * NX) {
      const unsigned q = r / NX;
      J = q < 3 ? q : NY - 6 + q;
      I = r - q * NX;
    } else {
      const unsigned r2 = r - 6 * NX, cc = r2 % 6;
      J = 3 + r2 / 6;
      I = cc < 3 ? cc : NX - 6 + cc;
    }
  }
  i = (int)I - 2;
  j = (int)J - 2;
  k = (int)K - 2;
}

// The nodes of the padded box within L layers of its faces (the two ghost
// layers, the boundary layer and L - 3 interior layers), enumerated as
// shell_node does for L = 3.
__host__ __device__ __forceinline__ long long thick_shell_count(const DevCfg &c, int L) {
  const long long NX = c.mx + 4, NY = c.my + 4, NZ = c.mz + 4;
  return 2LL * L * NX * NY + (NZ - 2LL * L) * (2LL * L * NX + 2LL * L * (NY - 2LL * L));
}
__host__ __device__ __forceinline__ void thick_shell_node(const DevCfg &c, int L, long long t64, int &i, int &j, int &k) {
  const unsigned t = (unsigned)t64;
  const unsigned L2 = 2u * L, NX = c.mx + 4, NY = c.my + 4, NZ = c.mz + 4, A = NX * NY, Pm = L2 * NX + L2 * (NY - L2);
  unsigned I, J, K;
  if (t < L2 * A) {
    const unsigned p = t / A, r = t - p * A;
    K = p < (unsigned)L ? p : NZ - L2 + p;
    J = r / NX;
    I = r - J * NX;
  } else {
    const unsigned t2 = t - L2 * A;
    K = L + t2 / Pm;
    const unsigned r = t2 - (K - L) * Pm;
    if (r < L2 * NX) {
      const unsigned q = r / NX;
      J = q < (unsigned)L ? q : NY - L2 + q;
      I = r - q * NX;
    } else {
      const unsigned r2 = r - L2 * NX, cc = r2 % L2;
      J = L + r2 / L2;
      I = cc < (unsigned)L ? cc : NX - L2 + cc;
    }
  }
  i = (int)I - 2;
  j = (int)J - 2;
  k = (int)K - 2;
}

// Copy of the planes' nodes within L layers of the faces (the part of a state
// FormBCS reads: periodic images two nodes across, face codes two nodes in).
static __global__ void thick_shell_copy_kernel(const DevCfg c, int L, const double *const *src, double *const *dst,
                                               int nplanes) {
  const long long total = thick_shell_count(c, L);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    thick_shell_node(c, L, t, i, j, k);
    const long long g = gidx(c, i, j, k);
    for (int p = 0; p < nplanes; p++) dst[p][g] = src[p][g];
  }
}

// Writes every non-interior node (boundary layer + both ghost layers) of qout.
static __global__ void bc_periodic_kernel(const DevCfg c, DevFields F) {
  const long long total = shell_count(c);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    shell_node(c, t, i, j, k);
    int si, sj, sk;
    bool from_in;
    bc_source(c, i, j, k, si, sj, sk, from_in);
    const long long g = gidx(c, i, j, k), s = gidx(c, si, sj, sk);
#pragma unroll
    for (int q = 0; q < 5; q++) F.qout[q][g] = from_in ? F.q[q][s] : F.qout[q][s];
  }
}

// ------------------------------------------------ non-periodic FormBCS --
// Blocks with boundary codes other than 7 (FormBCS rhs.c:477-1227), after the
// stage kernel has updated the interior: (1) the RK update of the boundary
// layer itself (the reference combines the whole global vector; Rhs is zero
// there), (2) the face codes in the reference's order i, j, k, (3) the
// periodic copies of the periodic directions from the stale stage input,
// (4) the ghost wrap.  Pressures are the stage input's EOS (lP before
// EqOfState refreshes it).

// (1) owned non-interior nodes: istage 0 Qold + adt*0, else beta Qold + adt*0 + alfa Qin
static __global__ void bc_combine_kernel(const DevCfg c, DevFields F, int istage, double alfa, double beta, double adt) {
  const long long total = shell_count(c);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    shell_node(c, t, i, j, k);
    if (i < 0 || i >= c.mx || j < 0 || j >= c.my || k < 0 || k >= c.mz) continue;
    const long long n = gidx(c, i, j, k);
#pragma unroll
    for (int q = 0; q < 5; q++) {
      const double qo = F.qold[q][n];
      F.qout[q][n] = (istage == 0) ? qo + adt * 0.0 : beta * qo + adt * 0.0 + alfa * F.q[q][n];
    }
  }
}

// user->ti of the step about to run: the time loop advances it before
// each step (main.c:887-974); the k-lo inflow code 47 reads it on the device
static __global__ void step_index_advance_kernel(int *ti) { *ti += 1; }

__device__ __forceinline__ double lp_at(const DevCfg &c, const DevFields &F, long long n) {
  if (F.pin) return F.pin[n];  // the pressure carried in lP
  const double r = F.q[0][n];
  return r != 0.0 ? (c.gamma - 1) * (F.q[4][n] - 0.5 * (F.q[1][n] * F.q[1][n] + F.q[2][n] * F.q[2][n] + F.q[3][n] * F.q[3][n]) / r)
                  : 0.0;
}

// (2) one direction's two faces; a thread per face node (lo and hi, as the
// reference's loop body)
static __global__ void bc_face_kernel(const DevCfg c, DevFields F, int dir, double alfa) {
  double *const *q = F.qout;
  const int *bc = c.bctype;
  const double g = c.gamma, Ma = c.ma;
  const long long si = 1, sj = c.px, sk = (long long)c.px * c.py;
  int na, nb, a0 = 0;
  if (dir == 0) { na = c.my; nb = c.mz; }
  else if (dir == 1) { na = c.mx; nb = c.mz; }
  else { na = c.mx; a0 = (bc[2] == 1) ? 1 : 0; nb = ((bc[3] == 1) ? c.my - 1 : c.my) - a0; }
  const long long total = (long long)na * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t % na), b = (int)(t / na);
    if (dir == 0) {  // rhs.c:601-636: j = a, k = b
      long long n = gidx(c, 0, a, b);
      if (bc[0] == 3) {
        q[0][n] = q[0][n + si]; q[1][n] = 0.; q[2][n] = q[2][n + si]; q[3][n] = q[3][n + si]; q[4][n] = q[4][n + si];
      } else if (bc[0] == 51) {
        q[0][n] = 0.445; q[1][n] = 0.311; q[2][n] = 0.; q[3][n] = 0.; q[4][n] = 8.928;
      }
      n = gidx(c, c.mx - 1, a, b);
      if (bc[1] == 3) {
        q[0][n] = q[0][n - si]; q[1][n] = 0.; q[2][n] = q[2][n - si]; q[3][n] = q[3][n - si]; q[4][n] = q[4][n - si];
      } else if (bc[0] == 51) {  // the high-i Lax state is keyed on bctype[0] (rhs.c:627)
        q[0][n] = 0.5; q[1][n] = 0.; q[2][n] = 0.; q[3][n] = 0.; q[4][n] = 1.4275;
      }
    } else if (dir == 1) {  // rhs.c:639-835: i = a, k = b
      long long n = gidx(c, a, 0, b);
      if (bc[2] == 3) {
        q[0][n] = q[0][n + sj]; q[1][n] = q[1][n + sj]; q[2][n] = 0.; q[3][n] = q[3][n + sj]; q[4][n] = q[4][n + sj];
      } else if (bc[2] == 10) {
        q[0][n] = q[0][n + sj]; q[1][n] = 0.; q[2][n] = q[2][n + sj]; q[3][n] = q[3][n + sj]; q[4][n] = q[4][n + sj];
      } else if (bc[2] == 1) {
        q[1][n] = 0.0; q[2][n] = 0.0; q[3][n] = 0.0;
        if (c.isothermal == 2 && alfa != 0 && F.nvert[n] < 1.5) {
          // characteristic isothermal wall (Poinsot & Lele), one pass (rhs.c:663-733, itr_tmp 1)
          const double *const *lq = F.q;
          const double ex = F.met[1][0][n], ey = F.met[1][1][n], ez = F.met[1][2][n];
          const double a_sound = sqrt(c.twall / (Ma * Ma));
          const double beta = sqrt(ey * ey + ex * ex + ez * ez);
          const double L0 = -a_sound * beta;
          if (!(b == 0 || b == c.mz - 1)) {
            const long long n1 = n + sj, n2 = n + 2 * sj;
            const double ajc = F.aj[n];
            double L = L0 * ajc *
                       ((-0.5 * lp_at(c, F, n2) + 2 * lp_at(c, F, n1) - 1.5 * lp_at(c, F, n)) -
                        lq[0][n] * a_sound / beta *
                            (ey * (-0.5 * lq[2][n2] / lq[0][n2] + 2. * lq[2][n1] / lq[0][n1] - 1.5 * lq[2][n] / lq[0][n]) +
                             ez * (-0.5 * lq[3][n2] / lq[0][n2] + 2. * lq[3][n1] / lq[0][n1] - 1.5 * lq[3][n] / lq[0][n])));
            if (c.twod != 1)
              L -= L0 * ajc * lq[0][n] * a_sound / beta * ex *
                   (-0.5 * lq[1][n2] / lq[0][n2] + 2. * lq[1][n1] / lq[0][n1] - 1.5 * lq[1][n] / lq[0][n]);
            q[0][n] = F.qold[0][n] - c.dt * alfa * L / a_sound / a_sound;
          }
        } else {
          const double lpn = lp_at(c, F, n + sj);
          q[0][n] = lpn * (g * Ma * Ma);
          q[4][n] = lpn / (g - 1);
        }
      }
      n = gidx(c, a, c.my - 1, b);
      if (bc[3] == 3) {
        q[0][n] = q[0][n - sj]; q[1][n] = q[1][n - sj]; q[2][n] = 0.; q[3][n] = q[3][n - sj]; q[4][n] = q[4][n - sj];
      } else if (bc[3] == 10) {
        q[0][n] = q[0][n - sj]; q[1][n] = 0.; q[2][n] = q[2][n - sj]; q[3][n] = q[3][n - sj]; q[4][n] = q[4][n - sj];
      } else if (bc[3] == 1) {
        q[1][n] = 0.0; q[2][n] = 0.0; q[3][n] = 0.0;
        if (c.isothermal == 2) {  // rhs.c:803-818
          const double *const *lq = F.q;
          const long long m1 = n - sj, m2 = n - 2 * sj;
          const double lp1 = lp_at(c, F, m1);
          const double a_sound = sqrt(g * lp1 / lq[0][m1]);
          const double L0 = lq[2][m1] / lq[0][m1] - a_sound;
          double L;
          if (b == 0 || b == c.mz - 1 || L0 > 0.) L = 0.;
          else
            L = L0 * F.aj[m1] * F.met[1][1][m1] *
                ((lp1 - lp_at(c, F, m2)) - lq[0][m1] * a_sound * (lq[2][n] / lq[0][n] - lq[2][m1] / lq[0][m1]));
          q[0][n] = F.qold[0][n] - c.dt * alfa * L / a_sound / a_sound;
          q[4][n] = q[0][n] * c.twall / (g * Ma * Ma) / (g - 1.0);
        } else {
          if (c.isothermal == 1) q[0][n] = lp_at(c, F, n) * (g * Ma * Ma);
          else q[0][n] = q[0][n - sj];
          q[4][n] = lp_at(c, F, n - sj) / (g - 1.0);
        }
      }
    } else {  // rhs.c:840-1087: i = a, j = a0 + b
      const int j = a0 + b;
      long long n = gidx(c, a, j, 0);
      if (bc[4] == 3) {
        q[0][n] = q[0][n + sk]; q[1][n] = q[1][n + sk]; q[2][n] = q[2][n + sk]; q[3][n] = 0.; q[4][n] = q[4][n + sk];
      } else if (bc[4] == 55) {  // u = Ma, rho = gamma (rhs.c:837)
        const double rho = g, u = Ma;
        q[0][n] = rho; q[3][n] = rho * u; q[4][n] = 0.5 * rho * u * u + 1. / (g - 1.);
      } else if (bc[4] == 44) {
        q[0][n] = q[0][n + sk]; q[1][n] = 0.; q[2][n] = 0.; q[3][n] = q[3][n + sk]; q[4][n] = q[4][n + sk];
      } else if (bc[4] == 45) {
        q[0][n] = 1.; q[3][n] = 1.; q[4][n] = .5 + 1. / (Ma * Ma * g * (g - 1.));
      } else if (bc[4] == 51) {
        q[0][n] = 0.445; q[3][n] = 0.311; q[4][n] = 8.928;
      } else if (bc[4] == 10) {
        q[0][n] = 1.; q[1][n] = 0.; q[2][n] = 0.; q[3][n] = 1.; q[4][n] = 1. / 0.4 + 0.5;
      } else if (bc[4] == 52) {
        // characteristic inlet imposing w = cos^2(pi/2 (y - 1)) (rhs.c:854-874),
        // with FormBCS's own truncated pi (rhs.c:488)
        const double pi = 3.14159265;
        const double *const *lq = F.q;
        const long long n1 = n + sk, n2 = n + 2 * sk;
        const double yy = F.cy[n];
        const double AA = cos(pi / 2 * (yy - 1.)) * cos(pi / 2 * (yy - 1.));
        const double lp1 = lp_at(c, F, n1), lp2 = lp_at(c, F, n2);
        const double a_sound = sqrt(g * lp1 / lq[0][n1]);
        const double Lam0 = lq[3][n1] / lq[0][n1] - a_sound;
        const double L0 = Lam0 * F.aj[n1] * F.met[2][2][n1] * ((lp2 - lp1) - lq[0][n1] * a_sound * (lq[3][n1] / lq[0][n1] - AA));
        const double L1 = (g - 1.) * L0, L4 = L0;
        const double d0 = 1. / (a_sound * a_sound) * (L1 + 0.5 * (L4 + L0));
        q[0][n] = F.qold[0][n] - c.dt * alfa * d0;
        const double lpn = q[0][n] / (g * Ma * Ma);
        q[3][n] = q[0][n] * AA;
        q[1][n] = 0.;
        q[2][n] = 0.;
        q[4][n] = 0.5 * q[3][n] * q[3][n] / q[0][n] + lpn / (g - 1);
      } else if (bc[4] == 47) {
        // power-law inflow with travelling perturbations in x and time
        // (rhs.c:904-950); ti: the running step's index
        const double pi = 3.141592;
        const double c1 = 0.03, c2 = -0.0032, c3 = 0.02, c4 = -0.01, yp1 = 1.0, yp2 = 1.5, yp3 = 2.0;
        const double w0 = 0.1, w1 = 0.25, w2 = 0.125, w3 = 0.0625;
        const double phi1 = 0.0, phi2 = 0.1, phi3 = 0.15, b0 = 0.5 * pi, b1 = 0.75 * pi, b2 = 0.5 * pi, b3 = 0.25 * pi;
        const double yy = F.cy[n], xx = F.cx[n];
        const double yplus = yy * 0.065 * c.ren;
        const int ti = *F.ti;
        if (yy < 8.0) {
          q[3][n] = pow(yy / 8.0, 0.1428);
        } else {
          q[3][n] = 1.0;
          q[1][n] = 0.0;
        }
        if (yy < 8.0) {
          q[3][n] += c1 * yplus * exp(-yplus / 12.5) * sin(w0 * ti * c.dt) * cos(b0 * xx);
          q[2][n] = c2 * yplus * yplus * exp(-yplus * yplus / 12.5 / 12.5) * sin(w0 * ti * c.dt) * cos(b0 * xx);
        } else if (yy >= 8.0) {
          q[3][n] += c3 * yy / yp1 * exp(-yy / yp1) * sin(w1 * ti * c.dt) * cos(b1 * xx + phi1) +
                     c3 * yy / yp2 * exp(-yy / yp2) * sin(w2 * ti * c.dt) * cos(b2 * xx + phi2) +
                     c3 * yy / yp3 * exp(-yy / yp3) * sin(w3 * ti * c.dt) * cos(b3 * xx + phi3);
          q[2][n] = c4 * yy * yy / yp1 / yp1 * exp(-yy * yy / yp1 / yp1) * sin(w1 * ti * c.dt) * cos(b1 * xx + phi1) +
                    c4 * yy * yy / yp2 / yp2 * exp(-yy * yy / yp2 / yp2) * sin(w2 * ti * c.dt) * cos(b2 * xx + phi2) +
                    c4 * yy * yy / yp3 / yp3 * exp(-yy * yy / yp3 / yp3) * sin(w3 * ti * c.dt) * cos(b3 * xx + phi3);
        }
        q[0][n] = 1.0;
        q[4][n] = 0.5 * q[3][n] * q[3][n] + 1. / (Ma * Ma * g * (g - 1.));
      }
      n = gidx(c, a, j, c.mz - 1);
      const long long m1 = n - sk, m2 = n - 2 * sk;
      if (bc[5] == 3) {
        q[0][n] = q[0][m1]; q[1][n] = q[1][m1]; q[2][n] = q[2][m1]; q[3][n] = 0.; q[4][n] = q[4][m1];
      } else if (bc[5] == 44) {
        q[0][n] = q[0][m1]; q[1][n] = 0.; q[2][n] = 0.; q[3][n] = q[3][m1]; q[4][n] = q[4][m1];
      } else if (bc[5] == 45) {
        q[0][n] = q[0][m1]; q[1][n] = q[1][m1]; q[2][n] = q[2][m1]; q[3][n] = q[3][m1]; q[4][n] = q[4][m1];
      } else if (bc[5] == 49) {  // characteristic (rhs.c:1003-1042)
        double Vn, Rplus, Rminus, sv, pOverrho, pp;
        const double lp1 = lp_at(c, F, m1);
        Vn = q[3][m1] / q[0][m1];
        double a_sound = sqrt(g * lp1 / q[0][m1]);
        const double lambda1 = Vn + a_sound, lambda2 = Vn - a_sound;
        if (Vn < 0.) {
          if (lambda1 < 0) {
            q[1][n] = 0.; q[2][n] = 0.;
            Rplus = Vn + 2 / Ma / (g - 1.);
            Rminus = Vn - 2 / Ma / (g - 1.);
            sv = 1. / (Ma * Ma * g);
          } else {
            Rplus = Vn + 2 * a_sound / (g - 1.);
            Rminus = Vn - 2 / Ma / (g - 1.);
            q[1][n] = 0.; q[2][n] = 0.;
            sv = 1. / (Ma * Ma * g);
          }
        } else {
          if (lambda2 >= 0) {
            Rplus = Vn + 2 * a_sound / (g - 1.);
            Rminus = Vn - 2 * a_sound / (g - 1.);
            q[1][n] = q[1][m1];
            q[2][n] = q[0][m1];  // rhoV takes rho (rhs.c:1022)
            sv = lp1 / pow(q[0][m1], g);
          } else {
            Rminus = Vn - 2 / Ma / (g - 1.);
            Rplus = Vn + 2 * a_sound / (g - 1.);
            q[1][n] = q[1][m1]; q[2][n] = q[2][m1];
            sv = lp1 / pow(q[0][m1], g);
          }
        }
        Vn = 0.5 * (Rplus + Rminus);
        a_sound = 0.25 * (g - 1.) * (Rplus - Rminus);
        pOverrho = a_sound * a_sound / (g);
        q[0][n] = pow(pOverrho / sv, 1. / (g - 2.));  // gamma-2 (rhs.c:1036)
        q[3][n] = q[0][n] * Vn;
        pp = pOverrho * q[0][n];
        q[4][n] = pp / (g - 1.) + 0.5 * (q[1][n] * q[1][n] + q[2][n] * q[2][n] + q[3][n] * q[3][n]) * q[0][n];
      } else if (bc[5] == 51) {
        q[0][n] = 0.5; q[1][n] = 0.; q[2][n] = 0.; q[3][n] = 0.; q[4][n] = 1.4275;
      } else if (bc[5] == 10) {
        q[0][n] = 1.; q[1][n] = 0.; q[2][n] = 0.; q[3][n] = 1.; q[4][n] = 1 / 0.4 + 0.5;
      } else if (bc[5] == 8) {  // subsonic non-reflecting outflow (rhs.c:1056-1086)
        const double *const *lq = F.q;
        const double lpn = lp_at(c, F, n), lp1 = lp_at(c, F, m1), lp2 = lp_at(c, F, m2);
        const double a_sound = sqrt(g * lp1 / lq[0][m1]);
        const double AA = q[3][m1] / q[0][m1];
        const double Lam0 = AA - a_sound, Lam4 = AA + a_sound;
        (void)Lam0;
        const double L0 = 0;
        const double L1 = AA * F.aj[m1] * F.met[2][2][m1] * (a_sound * a_sound * (lq[0][m1] - lq[0][m2]) - (lpn - lp1));
        const double L2 = AA * F.aj[m1] * F.met[2][2][m1] * (lq[1][m1] / q[0][m1] - lq[1][m2] / q[0][m1]);
        const double L3 = AA * F.aj[m1] * F.met[2][2][m1] * (lq[2][m1] / q[0][m1] - lq[2][m2] / q[0][m2]);
        const double L4 = Lam4 * F.aj[m1] * F.met[2][2][m1] *
                          ((lp1 - lp2) + q[0][m1] * a_sound * (lq[3][m1] / q[0][m1] - lq[3][m2] / q[0][m2]));
        (void)L2; (void)L3;
        const double d0 = 1. / (a_sound * a_sound) * (L1 + 0.5 * (L4 + L0));
        const double d1 = 0.5 * (L0 + L4);
        const double d2 = 0.5 / (q[0][m1] * a_sound) * (L4 - L0);
        q[0][n] = F.qold[0][n] - c.dt * alfa * d0;
        q[4][n] = F.qold[4][n] - c.dt * alfa *
                                     (0.5 * d0 * (lq[3][m1] / q[0][m1] * lq[3][m1] / q[0][m1]) + d1 / (g - 1.) +
                                      lq[3][m1] * d2);
        q[3][n] = F.qold[3][n] - c.dt * alfa * (lq[3][m1] / q[0][m1] * d0 + q[0][m1] * d2);
      }
    }
  }
}

// (3) periodic copies of one periodic direction with the reference's guards
// (i faces: 0 < k, 0 < j; j faces: j = 0 for k > 0, j = my-1 for 0 < k < mz-1;
// k faces unguarded), from the stale ghosted stage input.
static __global__ void bc_periodic_dir_kernel(const DevCfg c, DevFields F, int dir) {
  int na, nb;
  if (dir == 0) { na = c.my; nb = c.mz; }
  else if (dir == 1) { na = c.mx; nb = c.mz; }
  else { na = c.mx; nb = c.my; }
  const long long s = gstride(c, dir);
  const long long total = (long long)na * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t % na), b = (int)(t / na);
    long long lo, hi;
    bool do_lo = true, do_hi = true;
    if (dir == 0) {
      lo = gidx(c, 0, a, b); hi = gidx(c, c.mx - 1, a, b);
      do_lo = do_hi = (a > 0 && b > 0);
    } else if (dir == 1) {
      lo = gidx(c, a, 0, b); hi = gidx(c, a, c.my - 1, b);
      do_lo = b > 0;
      do_hi = b > 0 && b < c.mz - 1;
    } else {
      lo = gidx(c, a, b, 0); hi = gidx(c, a, b, c.mz - 1);
    }
#pragma unroll
    for (int q = 0; q < 5; q++) {
      if (do_lo) F.qout[q][lo] = F.q[q][lo - 2 * s];
      if (do_hi) F.qout[q][hi] = F.q[q][hi + 2 * s];
    }
  }
}

// The pressure's periodic copies in FormBCS (rhs.c:1107-1227 copy P from lP
// beside Q from lQ): fully periodic, the final value source of bc_source;
// `psnap` is P before the copies.
static __global__ void bc_periodic_p_kernel(const DevCfg c, const double *psnap, double *P) {
  const long long total = shell_count(c);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    shell_node(c, t, i, j, k);
    int si, sj, sk;
    bool from_in;
    bc_source(c, i, j, k, si, sj, sk, from_in);
    const long long g = gidx(c, i, j, k), s = gidx(c, si, sj, sk);
    P[g] = from_in ? psnap[s] : P[s];
  }
}

// One periodic direction's pressure copies with the guards of
// bc_periodic_dir_kernel.
static __global__ void bc_periodic_dir_p_kernel(const DevCfg c, const double *psnap, double *P, int dir) {
  int na, nb;
  if (dir == 0) { na = c.my; nb = c.mz; }
  else if (dir == 1) { na = c.mx; nb = c.mz; }
  else { na = c.mx; nb = c.my; }
  const long long s = gstride(c, dir);
  const long long total = (long long)na * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t % na), b = (int)(t / na);
    long long lo, hi;
    bool do_lo = true, do_hi = true;
    if (dir == 0) {
      lo = gidx(c, 0, a, b); hi = gidx(c, c.mx - 1, a, b);
      do_lo = do_hi = (a > 0 && b > 0);
    } else if (dir == 1) {
      lo = gidx(c, a, 0, b); hi = gidx(c, a, c.my - 1, b);
      do_lo = b > 0;
      do_hi = b > 0 && b < c.mz - 1;
    } else {
      lo = gidx(c, a, b, 0); hi = gidx(c, a, b, c.mz - 1);
    }
    if (do_lo) P[lo] = psnap[lo - 2 * s];
    if (do_hi) P[hi] = psnap[hi + 2 * s];
  }
}

// EqOfState (rhs.c:4820-4862) on every node of the padded box; rho = 0
// (unused padding) gives 0.
static __global__ void eos_plane_kernel(const DevCfg c, const double *const *q, double *P) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < c.plane; t += (long long)gridDim.x * blockDim.x) {
    const double r = q[0][t];
    P[t] = r != 0.0 ? (c.gamma - 1) * (q[4][t] - 0.5 * (q[1][t] * q[1][t] + q[2][t] * q[2][t] + q[3][t] * q[3][t]) / r)
                    : 0.0;
  }
}

// Ghost layers of periodic planes from their owned images (DMGlobalToLocal).
static __global__ void ghost_fill_kernel(const DevCfg c, double *const *planes, int nplanes) {
  const long long total = shell_count(c);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    shell_node(c, t, i, j, k);
    const bool gi = i < 0 || i >= c.mx, gj = j < 0 || j >= c.my, gk = k < 0 || k >= c.mz;
    if (!(gi || gj || gk)) continue;
    const bool pi = c.bctype[0] == 7, pj = c.bctype[2] == 7, pk = c.bctype[4] == 7;
    if ((gi && !pi) || (gj && !pj) || (gk && !pk)) continue;
    const long long g = gidx(c, i, j, k), s = gidx(c, wrapi(i, c.mx), wrapi(j, c.my), wrapi(k, c.mz));
    for (int p = 0; p < nplanes; p++) planes[p][g] = planes[p][s];
  }
}

// Compute_eddy_viscosity_LES (les.c:1523-1567) with constant CS
// (les.c:135-150) or, with csp, the dynamic model's CS per node: interior
// nodes only; velocity from the recorded state qu (nullptr: zero velocity
// before the first CalcUCat) or, with qn, as the dynamic model left lUcat.
// A block owns an EDDY_BX x EDDY_BY column of interior nodes and marches
// along k through a chunk of planes; the velocity u = rhoU / rho of three
// planes (k-1, k, k+1, with a one-node halo in i and j) sits in shared
// memory, so each node's three divisions happen once instead of at each of
// its six neighbours (the same IEEE quotients the reference forms there).
// nvert nullptr: nvert is zero everywhere (no immersed body).  The node's
// metrics, aj, filter width and nvert are loaded before the plane barrier so
// their latency overlaps the velocity conversion of the next plane.
constexpr int EDDY_BX = 32, EDDY_BY = 8, EDDY_PX = EDDY_BX + 2, EDDY_PN = EDDY_PX * (EDDY_BY + 2);
static __global__ void __launch_bounds__(EDDY_BX *EDDY_BY, 4)
    eddy_viscosity_kernel(const DevCfg c, const double *const *qu, const double *const *met, const double *aj,
                          const double *delta2, const double *nvert, double *nut, int kchunk,
                          const double *const *qn = nullptr, const double *csp = nullptr) {
  __shared__ double us[3][3][EDDY_PN];  // [slot][component][node]
  __shared__ double stq[4][EDDY_PN];    // raw rho, rhoU, rhoV, rhoW of the plane in flight
  __shared__ unsigned char stv[EDDY_PN];  // the staged node's velocity source: 0 none, 1 qu, 2 qn
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * EDDY_BX + tx;
  const int i0 = 1 + blockIdx.x * EDDY_BX, j0 = 1 + blockIdx.y * EDDY_BY;
  const int kb = 1 + blockIdx.z * kchunk, ke = min(c.mz - 1, kb + kchunk);
  const int i = i0 + tx, j = j0 + ty;
  const bool act = i <= c.mx - 2 && j <= c.my - 2;
  // asynchronous copy of plane kk's raw state into the staging area (halo
  // entries beyond the owned nodes get no source and stay zero velocity)
  auto issue = [&](int kk) {
    for (int e = tid; e < EDDY_PN; e += EDDY_BX * EDDY_BY) {
      const int ly = e / EDDY_PX, lx = e - ly * EDDY_PX;
      const int xi = i0 - 1 + lx, yj = j0 - 1 + ly;
      const double *const *src = nullptr;
      long long n = 0;
      unsigned char sv = 0;
      if (xi <= c.mx - 1 && yj <= c.my - 1) {
        n = gidx(c, xi, yj, kk);
        src = qu;
        sv = qu ? 1 : 0;
        // after the dynamic model (qn set) lUcat holds the current state's
        // velocity at interior nodes with nvert <= 1.1 (les.c:234-238)
        if (qn && xi >= 1 && xi <= c.mx - 2 && yj >= 1 && yj <= c.my - 2 && kk >= 1 && kk <= c.mz - 2 &&
            (!nvert || ldg(nvert + n) <= 1.1)) {
          src = qn;
          sv = 2;
        }
      }
      const bool v = src != nullptr;
      stv[e] = sv;
#pragma unroll
      for (int f = 0; f < 4; f++) cp_async8(&stq[f][e], v ? src[f] + n : (const double *)nut, v);
    }
    cp_async_commit();
  };
  // staged plane -> velocity slot s: the same quotients as before
  auto convert = [&](int s) {
    for (int e = tid; e < EDDY_PN; e += EDDY_BX * EDDY_BY) {
      double u0 = 0., u1 = 0., u2 = 0.;
      if (stv[e]) {
        const double r = stq[0][e];
        // lUcat x = 0 with -twoD 1 (rhs.c:1349), except where the dynamic
        // model rewrote it from the state (les.c:255)
        u0 = (c.twod == 1 && stv[e] == 1) ? 0. : stq[1][e] / r;
        u1 = stq[2][e] / r;
        u2 = stq[3][e] / r;
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
  const int e0 = (ty + 1) * EDDY_PX + tx + 1;
  for (int k = kb; k < ke; k++) {
    // the node's own operands of plane k, in flight across the barriers
    const long long n = gidx(c, i, j, k);
    double mv[3][3], ajc = 0., d2 = 0., cs = 0.;
    bool solid = false;
    if (act) {
#pragma unroll
      for (int e = 0; e < 3; e++)
#pragma unroll
        for (int x = 0; x < 3; x++) mv[e][x] = ldg(met[e * 3 + x] + n);
      ajc = ldg(aj + n);
      d2 = ldg(delta2 + n);
      cs = csp ? ldg(csp + n) : c.cs_const;
      solid = nvert && ldg(nvert + n) > 0.1;
    }
    cp_async_wait_all();
    __syncthreads();  // plane k+1 staged; every thread is past plane k-1, whose slot (k+1) % 3 is refilled now
    convert((k + 1) % 3);
    __syncthreads();
    if (k + 1 < ke) issue(k + 2);  // in flight while plane k is computed
    if (act) {
      if (solid) {
        nut[n] = 0.;
      } else {
        const int sm = (k - 1) % 3, s0 = k % 3, sp = (k + 1) % 3;
        double dd[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
          dd[a][0] = (us[s0][a][e0 + 1] - us[s0][a][e0 - 1]) * 0.5;
          dd[a][1] = (us[s0][a][e0 + EDDY_PX] - us[s0][a][e0 - EDDY_PX]) * 0.5;
          dd[a][2] = (us[sp][a][e0] - us[sm][a][e0]) * 0.5;
        }
        double g[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int x = 0; x < 3; x++)
            g[a][x] = (dd[a][0] * mv[0][x] + dd[a][1] * mv[1][x] + dd[a][2] * mv[2][x]) * ajc;
        const double Sdd = 2. / 3. * (g[0][0] + g[1][1] + g[2][2]);
        const double Sxx = 0.5 * (g[0][0] + g[0][0]) - Sdd, Sxy = 0.5 * (g[0][1] + g[1][0]), Sxz = 0.5 * (g[0][2] + g[2][0]);
        const double Syy = 0.5 * (g[1][1] + g[1][1]) - Sdd, Syz = 0.5 * (g[1][2] + g[2][1]);
        const double Szz = 0.5 * (g[2][2] + g[2][2]) - Sdd;
        const double Sabs = sqrt(2.0 * (Sxx * Sxx + Sxy * Sxy + Sxz * Sxz + Sxy * Sxy + Syy * Syy + Syz * Syz +
                                        Sxz * Sxz + Syz * Syz + Szz * Szz));
        nut[n] = cs * d2 * Sabs;  // CS * pow(pow(1/aj,1/3),2) * |S|
      }
    }
  }
}
// k-chunk of the eddy-viscosity march: the fewest whole waves of resident
// blocks, each chunk paying two extra velocity planes (cost = waves x
// (chunk + 2)); the result does not depend on it
static inline int eddy_kchunk(const DevCfg &c, int sms) {
  static int resident = 0;  // blocks per SM, from the occupancy calculator once per process
  if (resident == 0) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, eddy_viscosity_kernel, EDDY_BX * EDDY_BY, 0) != cudaSuccess ||
        nb < 1)
      nb = 1;
    resident = nb;
  }
  const int nk = c.mz - 2;
  if (nk <= 4) return nk < 1 ? 1 : nk;
  const long long tiles = (long long)((c.mx - 2 + EDDY_BX - 1) / EDDY_BX) * ((c.my - 2 + EDDY_BY - 1) / EDDY_BY);
  const long long slots = (long long)(sms > 0 ? sms : 1) * resident;
  int best = nk;
  double bc = 1e300;
  for (int kc = 4; kc <= nk; kc++) {
    const long long blocks = tiles * ((nk + kc - 1) / kc);
    const double cost = (double)((blocks + slots - 1) / slots) * (kc + 2);
    if (cost < bc) { bc = cost; best = kc; }
  }
  return best;
}
static inline dim3 eddy_grid(const DevCfg &c, int kchunk) {
  return dim3((c.mx - 2 + EDDY_BX - 1) / EDDY_BX, (c.my - 2 + EDDY_BY - 1) / EDDY_BY, (c.mz - 2 + kchunk - 1) / kchunk);
}

// ------------------------------------------------------------ shock sensor --
// Hybrid weights with -calc_sigma (formConvectionLES at istage 0,
// rhs.c:3328-3433; compute_ri / sigma_cent rhs.c:2334-2358).  Three passes
// with a ghost fill between them, as the reference's DMGlobalToLocal calls:
// raw ramp per direction, product filter of neighbour square roots,
// curvature rule with y = z = min(y, z).  Boundary nodes keep (s_x, s_y, s_z).
__device__ __forceinline__ double sensor_ri(double fR, double f0, double fL, double ks) {
  const double dfL = fL - f0, dfR = f0 - fR;
  return (fabs(2 * dfL * dfR) + ks) / (dfL * dfL + dfR * dfR + ks);
}
__device__ __forceinline__ double sensor_ramp(double fL, double f0, double fR, double fRR, double ks) {
  const double rL = sensor_ri(fL, f0, fR, ks), rR = sensor_ri(f0, fR, fRR, ks);
  const double r = (rR < rL) ? rR : rL;
  const double rd = 0.5;
  const double rmax = (rd < r) ? r : rd;
  return 0.5 + 0.5 * tanh(3.0 * (r - rd) / rmax) / tanh(3.0);
}
__device__ __forceinline__ double eos_node(const DevCfg &c, const double *const *q, long long n) {
  const double r = q[0][n];
  return r != 0.0 ? (c.gamma - 1) * (q[4][n] - 0.5 * (q[1][n] * q[1][n] + q[2][n] * q[2][n] + q[3][n] * q[3][n]) / r)
                  : 0.0;
}
__device__ __forceinline__ double pmin(double a, double b) { return (a < b) ? a : b; }
__device__ __forceinline__ double pmax(double a, double b) { return (a < b) ? b : a; }

// pass 1: every node (s_x, s_y, s_z); interior nodes the clipped ramp of p:
// the plane P when given (the pressure an immersed step carries into the next
// step's first stage, which formConvectionLES reads as lP), else the EOS of q
__device__ __forceinline__ double sensor_p(const DevCfg &c, const double *const *q, const double *P, long long n) {
  return P ? P[n] : eos_node(c, q, n);
}
static __global__ void sigma_sensor_kernel(const DevCfg c, const double *const *q, double *const *sig,
                                           const double *P) {
  const long long total = (long long)c.px * c.py * c.pz;
  const long long si = 1, sj = c.px, sk = (long long)c.px * c.py;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % c.px) - 2, j = (int)((t / c.px) % c.py) - 2, k = (int)(t / sk) - 2;
    double sx = c.s_x, sy = c.s_y, sz = c.s_z;
    if (i >= 1 && i <= c.mx - 2 && j >= 1 && j <= c.my - 2 && k >= 1 && k <= c.mz - 2) {
      const long long n = t;
      const double p0 = sensor_p(c, q, P, n);
      const bool absorb = c.abc != 0 && k > c.abc;  // -ABC layer: raw weight 0 (rhs.c:3341, 3355, 3368)
      if (absorb) sx = 0.;
      else if (i < c.mx - 4 && i > 2)
        sx = sensor_ramp(sensor_p(c, q, P, n - si), p0, sensor_p(c, q, P, n + si), sensor_p(c, q, P, n + 2 * si), c.ks);
      sx = pmax(c.s_x_min, pmin(c.s_x, sx));
      if (absorb) sz = 0.;
      else if (c.bctype[4] == 7 || (k < c.mz - 4 && k > 4))
        sz = sensor_ramp(sensor_p(c, q, P, n - sk), p0, sensor_p(c, q, P, n + sk), sensor_p(c, q, P, n + 2 * sk), c.ks);
      sz = pmax(c.s_z_min, pmin(c.s_z, sz));
      if (absorb) sy = 0.;
      else if (j < c.my - 4 && j > 4)
        sy = sensor_ramp(sensor_p(c, q, P, n - sj), p0, sensor_p(c, q, P, n + sj), sensor_p(c, q, P, n + 2 * sj), c.ks);
      sy = pmax(c.s_y_min, pmin(c.s_y, sy));
    }
    sig[0][t] = sx;
    sig[1][t] = sy;
    sig[2][t] = sz;
  }
}

// pass 2 (ls: ghosted pass-1 planes): interior nodes times
// sqrt(ls[j-1] ls) sqrt(ls[k-1] ls[k+1]) sqrt(ls[i-1] ls[i+1]); others copied
static __global__ void sigma_filter_kernel(const DevCfg c, const double *const *ls, double *const *sig) {
  const long long total = (long long)c.px * c.py * c.pz;
  const long long si = 1, sj = c.px, sk = (long long)c.px * c.py;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % c.px) - 2, j = (int)((t / c.px) % c.py) - 2, k = (int)(t / sk) - 2;
    const bool inner = i >= 1 && i <= c.mx - 2 && j >= 1 && j <= c.my - 2 && k >= 1 && k <= c.mz - 2;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double *l = ls[a];
      double v = l[t];
      if (inner) v *= sqrt(l[t - sj] * l[t]) * sqrt(l[t - sk] * l[t + sk]) * sqrt(l[t - si] * l[t + si]);
      sig[a][t] = v;
    }
  }
}

// pass 3 (ls: ghosted pass-2 planes): curvature rule, then y = z = min(z, y)
static __global__ void sigma_post_kernel(const DevCfg c, const double *const *ls, double *const *sig) {
  const long long total = (long long)c.px * c.py * c.pz;
  const long long sj = c.px, sk = (long long)c.px * c.py;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % c.px) - 2, j = (int)((t / c.px) % c.py) - 2, k = (int)(t / sk) - 2;
    double x = ls[0][t], y = ls[1][t], z = ls[2][t];
    if (i >= 1 && i <= c.mx - 2 && j >= 1 && j <= c.my - 2 && k >= 1 && k <= c.mz - 2) {
      const double *ly = ls[1], *lz = ls[2];
      if (j < c.my - 4 && j > 4 && ly[t - sj] + ly[t + sj] - 2. * ly[t] < 0.0) y = (ly[t - sj] * ly[t] * ly[t]);
      if (k < c.mz - 4 && k > 4 && lz[t - sk] + lz[t + sk] - 2. * lz[t] < 0.0) z = (lz[t - sk] * lz[t + sk] * lz[t]);
      z = pmin(z, y);
      y = z;
    }
    sig[0][t] = x;
    sig[1][t] = y;
    sig[2][t] = z;
  }
}

// LES filter width squared per node, pow(pow(1/aj, 1/3), 2.0) -- the value
// formViscous (rhs.c:1694-1696) and Compute_eddy_viscosity_LES (les.c:1560-1561)
// recompute at every use; aj is fixed after FormMetrics, so once per grid.
static __global__ void delta2_kernel(const DevCfg c, const double *aj, double *delta2) {
  const long long total = (long long)c.px * c.py * c.pz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const double a = aj[t];
    delta2[t] = a != 0.0 ? pow(pow(1. / a, 1. / 3.), 2.0) : 0.0;
  }
}

// ---------------------------------------------------------------- metrics --
// FormMetrics (metrics.c:52-136): csi on (k,j) interior for every i, eta on
// (k,i) interior for every j, zet on (j,i) interior for every k, aj on the
// interior; everything else zero.
static __global__ void metrics_interior_kernel(const DevCfg c, const double *const *X, double *const *met, double *aj) {
  const long long nx = c.mx, ny = c.my, nz = c.mz, total = nx * ny * nz;
  const long long si = 1, sj = c.px, sk = (long long)c.px * c.py;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / (nx * ny));
    const long long n = gidx(c, i, j, k);
    const bool ii = i > 0 && i < c.mx - 1, jj = j > 0 && j < c.my - 1, kk = k > 0 && k < c.mz - 1;
    double dc[3], de[3], dz[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      dc[a] = ii ? 0.5 * (X[a][n + si] - X[a][n - si]) : 0.;
      de[a] = jj ? 0.5 * (X[a][n + sj] - X[a][n - sj]) : 0.;
      dz[a] = kk ? 0.5 * (X[a][n + sk] - X[a][n - sk]) : 0.;
    }
    double v[10];
    for (int a = 0; a < 10; a++) v[a] = 0.;
    if (kk && jj) {
      v[0] = de[1] * dz[2] - de[2] * dz[1];
      v[1] = -de[0] * dz[2] + de[2] * dz[0];
      v[2] = de[0] * dz[1] - de[1] * dz[0];
    }
    if (kk && ii) {
      v[3] = dz[1] * dc[2] - dz[2] * dc[1];
      v[4] = -dz[0] * dc[2] + dz[2] * dc[0];
      v[5] = dz[0] * dc[1] - dz[1] * dc[0];
    }
    if (jj && ii) {
      v[6] = dc[1] * de[2] - dc[2] * de[1];
      v[7] = -dc[0] * de[2] + dc[2] * de[0];
      v[8] = dc[0] * de[1] - dc[1] * de[0];
    }
    if (ii && jj && kk) {
      const double det = dc[0] * (de[1] * dz[2] - de[2] * dz[1]) - dc[1] * (de[0] * dz[2] - de[2] * dz[0]) +
                         dc[2] * (de[0] * dz[1] - de[1] * dz[0]);
      v[9] = 1. / det;
    }
    for (int a = 0; a < 9; a++) met[a][n] = v[a];
    aj[n] = v[9];
  }
}

// One boundary-copy pass of FormMetrics (metrics.c:138-246).  face: 0 i-lo,
// 1 i-hi, 2 j-lo, 3 j-hi, 4 k-lo, 5 k-hi.  The passes must run in this order.
static __global__ void metrics_boundary_kernel(const DevCfg c, double *const *met, double *aj, int face) {
  const int d = face / 2, hi = face & 1;
  const int na = d == 0 ? c.my : c.mx, nb = d == 2 ? c.my : c.mz;  // the two transverse extents
  const long long total = (long long)na * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t % na), b = (int)(t / na);
    int i, j, k;
    if (d == 0) { i = hi ? c.mx - 1 : 0; j = a; k = b; }
    else if (d == 1) { j = hi ? c.my - 1 : 0; i = a; k = b; }
    else { k = hi ? c.mz - 1 : 0; i = a; j = b; }
    const long long n = gidx(c, i, j, k);
    const long long s = hi ? -gstride(c, d) : gstride(c, d);
    // i faces copy eta,zet; j faces csi,zet; k faces eta,csi (plus aj always)
    const int m1 = d == 0 ? 1 : 0, m2 = d == 2 ? 1 : 2;
    for (int q = 0; q < 3; q++) {
      met[m1 * 3 + q][n] = met[m1 * 3 + q][n + s];
      met[m2 * 3 + q][n] = met[m2 * 3 + q][n + s];
    }
    aj[n] = aj[n + s];
  }
}

// --------------------------------------------------------- pack / unpack --
// AoS natural (mz,my,mx,nc) <-> owned nodes of nc padded planes.
static __global__ void unpack_kernel(const DevCfg c, const double *__restrict__ aos, int nc, double *const *planes) {
  const long long total = (long long)c.mx * c.my * c.mz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % c.mx), j = (int)((t / c.mx) % c.my), k = (int)(t / ((long long)c.mx * c.my));
    const long long g = gidx(c, i, j, k);
    for (int q = 0; q < nc; q++) planes[q][g] = aos[t * nc + q];
  }
}

static __global__ void pack_kernel(const DevCfg c, const double *const *planes, int nc, double *__restrict__ aos) {
  const long long total = (long long)c.mx * c.my * c.mz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % c.mx), j = (int)((t / c.mx) % c.my), k = (int)(t / ((long long)c.mx * c.my));
    const long long g = gidx(c, i, j, k);
    for (int q = 0; q < nc; q++) aos[t * nc + q] = planes[q][g];
  }
}

// EqOfState (rhs.c:4845-4856) on owned nodes, written AoS (1 per node).
static __global__ void eos_pack_kernel(const DevCfg c, const double *const *q, double *__restrict__ p) {
  const long long total = (long long)c.mx * c.my * c.mz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % c.mx), j = (int)((t / c.mx) % c.my), k = (int)(t / ((long long)c.mx * c.my));
    const long long g = gidx(c, i, j, k);
    const double r = q[0][g], ru = q[1][g], rv = q[2][g], rw = q[3][g], re = q[4][g];
    p[t] = (c.gamma - 1) * (re - 0.5 * (ru * ru + rv * rv + rw * rw) / r);
  }
}

}  // namespace cb

namespace cb {

// ------------------------------------------------------------------- CFL --
// Largest inviscid spectral radius over the interior nodes,
//   lambda = aj * sum_d ( |m_d . u| + c |m_d| ),  c^2 = gamma p / rho,
// with m_d the contravariant area vectors (csi, eta, zet carry 1/J), so that
// dt = CFL / lambda_max.  The reference keeps dt fixed (-dt, init.c:94) and its
// Spectral (rhs.c:4739-4814) is an unused incompressible estimate; this is the
// compressible one the time-step controller needs.  Max per warp by shuffles,
// per block through shared memory, one atomicMax per block on the bit pattern
// of the (non-negative) double.
static __global__ void spectral_radius_kernel(const DevCfg c, const double *const *q, const double *const *met,
                                              const double *aj, const double *nvert, unsigned long long *out) {
  const long long nx = c.mx - 2, ny = c.my - 2, nz = c.mz - 2, total = nx * ny * nz;
  double lmax = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % nx), j = 1 + (int)((t / nx) % ny), k = 1 + (int)(t / (nx * ny));
    const long long n = gidx(c, i, j, k);
    if (ldg(nvert + n) >= 0.1) continue;  // solid and interface nodes carry no RHS (rhs.c:4610)
    const double r = ldg(q[0] + n), u = ldg(q[1] + n) / r, v = ldg(q[2] + n) / r, w = ldg(q[3] + n) / r;
    const double p = (c.gamma - 1) * (ldg(q[4] + n) - 0.5 * r * (u * u + v * v + w * w));
    const double cs = sqrt(fabs(c.gamma * p / r));
    double lam = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double mx = ldg(met[3 * d] + n), my = ldg(met[3 * d + 1] + n), mz = ldg(met[3 * d + 2] + n);
      lam += fabs(mx * u + my * v + mz * w) + cs * sqrt(mx * mx + my * my + mz * mz);
    }
    lam *= ldg(aj + n);
    lmax = fmax(lmax, lam);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
  __shared__ double wmax[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) wmax[warp] = lmax;
  __syncthreads();
  if (warp == 0) {
    double m = lane < (int)(blockDim.x >> 5) ? wmax[lane] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));  // order-preserving for m >= 0
  }
}

}  // namespace cb
