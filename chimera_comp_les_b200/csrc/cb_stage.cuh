// Fused stage kernel: formRHS (inviscid + viscous + SGS face fluxes, flux
// difference, MultAj) followed by the SSP-RK stage combination.
//
// Reference arithmetic restated (rhs.c):
//   formConvection      2570-3224   (non-LES upwind: first order / MUSCL / WENO3, Rusanov)
//   formConvectionLES   3231-4291   (upwind blended with a 4-point central flux by sigma)
//   formViscous         1367-2254   (stress, heat flux, eddy viscosity, Yoshizawa, LES energy)
//   MultAj / formRHS    4575-4736
//   RungeKutta          solvers.c:232-271 (stage combination)
//
// Two forms share this code, selected by the flux type R:
//   R = double, MIX = false : the FP64 parity form, the reference's IEEE operation order.
//   R = float,  MIX = true  : the mixed form.  The state, the EOS and the RK combination
//     stay FP64; reconstruction, Riemann/central fluxes, viscous and SGS terms run in FP32.
//     FP64 -> FP32 rounding would erase the low-Mach pressure signal (p ~ 100, dp ~ 0.06),
//     so the FP64 EOS delivers p' = p - p_ref, rhoE' = rhoE - E_ref, T' = T - T_ref and the
//     FP32 fluxes carry only fluctuations.  The constant part p_ref*h of every momentum
//     face flux is restored exactly in FP64 through the per-node metric divergence
//     gcl = sum_d (h_d(+1/2) - h_d(-1/2)); the constant part H_ref = E_ref + p_ref of the
//     energy flux is carried in FP32 (its error is relative to H_ref * dU).
//
// Execution shape (B200): a block owns a 32 x BY column of interior nodes and
// marches along k through a chunk of planes.  A ring of node planes (k-1 ..
// k+2, each with a two-node halo in i and j; k-2 .. k+3 for the WENO5-JS
// variants) lives in shared memory holding the conserved state and the
// derived p, u, v, w, T=p/rho, so every division of the EOS / CalcUCat happens
// once per node.  Each face flux is computed exactly once per plane.
// Metrics, nvert and nu_t are read through the read-only cache.
#pragma once
#include "cb_common.cuh"

namespace cb {

constexpr int NF = 10;  // fields per node in the plane ring
enum { F_RHO = 0, F_RU, F_RV, F_RW, F_RE, F_P, F_U, F_V, F_W, F_T };

constexpr double BLANKWALL = 2.9;
constexpr double BLANK = 0.1;
constexpr double SOLID = 0.5;
constexpr double INNERBLANK = 7.;
constexpr double GAMMA_CONV = 1.4;  // formConvection[LES] fix gamma = 1.4 (rhs.c:2596, 3257)

// face buffer width: FP64 keeps conv (5), visc (5), LES stress (3) apart to
// difference them in the reference's order; the mixed form stores visc-conv.
template <bool MIX>
struct FaceWidth {
  static constexpr int NG = MIX ? 8 : 13;
  static constexpr int VOFF = MIX ? 0 : 5;   // visc offset
  static constexpr int AOFF = MIX ? 5 : 10;  // LES stress offset
};

template <int BX, int BY>
struct TileShape {
  static constexpr int PX = BX + 4, PY = BY + 4, PN = PX * PY;
  static constexpr int NXF = (BX + 1) * BY;
  static constexpr int NYF = BX * (BY + 1);
};

// FLUX bits of the stage kernel (see conv_face): Roe's flux, a constant LES
// blend weight of exactly 1 or 0, and WENO5-JS reconstruction.  FLUX_PLAIN
// (no-IBM variants): every face of the block is periodic or an interface
// (bctype 7 on all six sides), -twoD is 0, and without FLUX_W5 the
// reconstruction is MUSCL (fluxorder 2) -- the options the host checked, as
// compile-time constants, so the kernel carries no other branch of them.
constexpr int FLUX_ROE = 1, FLUX_SIGMA1 = 2, FLUX_SIGMA0 = 4, FLUX_W5 = 8, FLUX_PLAIN = 16;

// Tile geometry of a stage-kernel variant.  The WENO3/MUSCL stencil reaches
// one node beyond the face's two nodes: a ring of 4 planes (k-1 .. k+2) and a
// 32 x 7 tile of 256 threads.  WENO5-JS reaches two: a ring of 6 planes
// (k-2 .. k+3), which fits the shared memory of one block (FP64) or two
// (mixed) per SM with a 32 x 5 tile of 192 threads.  The i/j halo stays two
// nodes: the few stencil nodes beyond it are read from global memory.
template <int FLUX>
struct StageGeo {
  static constexpr bool W5 = (FLUX & FLUX_W5) != 0;
  static constexpr int BX = 32, BY = W5 ? 5 : 7, NT = BX * (BY + 1);
  static constexpr int NPL = W5 ? 6 : 4;  // ring planes
  static constexpr int H = W5 ? 2 : 1;    // ring planes below the current one
  using Tile = TileShape<BX, BY>;
  static constexpr int NXF = Tile::NXF, NYF = Tile::NYF, NZF = BX * BY;
  static_assert(NXF <= NT && NYF <= NT && NZF <= NT, "one face direction per round of the schedule");
};

// Threads of a stage-kernel block.  The FP64 form runs two threads per face:
// the first NT compute the faces' inviscid fluxes, the next NT their viscous
// and SGS fluxes, so each thread holds half the live FP64 values and a block
// of 2 NT threads fits the register file (16 warps per SM at 32 x 7 instead of
// 8).  The mixed form keeps one thread per face and two blocks per SM.
template <int FLUX, bool MIX>
struct StageThreads {
  static constexpr bool SPLIT = !MIX;
  static constexpr int N = StageGeo<FLUX>::NT * (SPLIT ? 2 : 1);
  static constexpr int MIN_BLOCKS = MIX ? 2 : 1;
};

// The mixed form's no-IBM MUSCL/WENO3 variants read the FP32 metric vectors
// and nu_t of the current plane from a shared-memory slot that the block
// fills with 16-byte cp.async copies one plane ahead of use, instead of about
// 18 metric loads per node through the L1; only the k-faces' far node (plane
// k+1) is still read from global memory.  The kernel reads the same values
// either way.
template <bool MIX, bool NV0, int FLUX>
struct StageMet {
  static constexpr bool on = MIX && NV0 && (FLUX & FLUX_W5) == 0;
};

// Selections by a runtime direction d without dynamic indexing (which would
// place the indexed array in local memory).
template <typename R>
__device__ __forceinline__ const R *met_ptr(const DevFields &F, int d, int q);
template <>
__device__ __forceinline__ const double *met_ptr<double>(const DevFields &F, int d, int q) {
  return d == 0 ? F.met[0][q] : (d == 1 ? F.met[1][q] : F.met[2][q]);
}

template <typename R>
__device__ __forceinline__ R ldr(const R *p) { return __ldg(p); }

// Metric vector of direction e at node g in the form's arithmetic type; w is
// the mixed form's companion value (FP32 filter width for e = 0, aj for e = 1).
template <typename R>
struct MetV {
  R x, y, z, w;
};
template <typename R, bool MIX>
__device__ __forceinline__ MetV<R> met_load(const DevFields &F, int e, long long g) {
  MetV<R> r;
  if constexpr (MIX) {
    const float4 v = __ldg((e == 0 ? F.met4[0] : (e == 1 ? F.met4[1] : F.met4[2])) + g);
    r.x = v.x; r.y = v.y; r.z = v.z; r.w = v.w;
  } else {
    r.x = ldg(met_ptr<double>(F, e, 0) + g);
    r.y = ldg(met_ptr<double>(F, e, 1) + g);
    r.z = ldg(met_ptr<double>(F, e, 2) + g);
    r.w = 0.;
  }
  return r;
}

__device__ __forceinline__ int bc_lo(const DevCfg &c, int d) { return d == 0 ? c.bctype[0] : (d == 1 ? c.bctype[2] : c.bctype[4]); }
__device__ __forceinline__ int bc_hi(const DevCfg &c, int d) { return d == 0 ? c.bctype[1] : (d == 1 ? c.bctype[3] : c.bctype[5]); }

struct NRef {
  int r, y, x;  // relative plane (-1..2), tile-local row, tile-local column
};

__device__ __forceinline__ NRef nshift(NRef n, int d, int s) {
  if (d == 0) n.x += s;
  else if (d == 1) n.y += s;
  else n.r += s;
  return n;
}

template <typename R, int BX, int BY, int NPL = 4>
struct Ring {
  static constexpr int PX = TileShape<BX, BY>::PX, PY = TileShape<BX, BY>::PY;
  static constexpr int H = (NPL - 2) / 2;  // ring planes below the current one
  R *pl;
  const unsigned char *nvc;  // [NPL][PN] nvert * 4 (exact when DevCfg::nvq)
  // mixed no-IBM variants (StageMet): the FP32 metric vectors [3][MPN] and
  // nu_t [MPN] of the current plane over the (BX+2) x (BY+2) node box that
  // starts one node before the tile in i and j (every face's two nodes)
  static constexpr int MPX = BX + 2, MPY = BY + 2, MPN = MPX * MPY;
  const float4 *mt;
  const double *nt;
  __device__ __forceinline__ float4 met(int e, NRef n) const { return mt[e * MPN + (n.y - 1) * MPX + (n.x - 1)]; }
  __device__ __forceinline__ double nut(NRef n) const { return nt[(n.y - 1) * MPX + (n.x - 1)]; }
  // slot of relative plane r (-H .. NPL-H-1) is sb + r + H modulo NPL, with
  // sb the slot of the lowest plane: a rotation, no table
  int sb;
  __device__ __forceinline__ int slot(int r) const {
    if constexpr (NPL == 4) return (sb + r + 1) & 3;
    const int t = sb + r + H;
    return t >= NPL ? t - NPL : t;
  }
  // FP64 form: field-major planes [slot][field][y][x] (consecutive x in
  // consecutive banks).  Mixed form: the NF fields of a node side by side
  // [slot][y][x][field], read in 8-byte pairs (fields 2m, 2m+1): a node's
  // state, pressure and velocity come in 5 loads instead of 10, and a warp's
  // 8-byte loads at the 40-byte node stride hit distinct banks.
  static constexpr bool AOS = sizeof(R) == 4;
  __device__ __forceinline__ R get(int f, NRef n) const {
    if constexpr (AOS) {
      const float2 v = *reinterpret_cast<const float2 *>(pl + ((slot(n.r) * PY + n.y) * PX + n.x) * NF + (f & ~1));
      return (f & 1) ? v.y : v.x;
    } else {
      return pl[((slot(n.r) * NF + f) * PY + n.y) * PX + n.x];
    }
  }
  __device__ __forceinline__ double nv(NRef n) const { return 0.25 * (double)nvc[(slot(n.r) * PY + n.y) * PX + n.x]; }
  // a node of the i/j halo rows the ring holds (the k range is always held)
  __device__ __forceinline__ bool holds(NRef n) const { return n.x >= 0 && n.x < PX && n.y >= 0 && n.y < PY; }
};

// nvert of a ring node: from shared memory when the byte code is exact, else
// from global memory at g
template <class RG>
__device__ __forceinline__ double nvert_at(const DevCfg &c, const DevFields &F, const RG &Rg, NRef n, long long g) {
  return c.nvq ? Rg.nv(n) : ldg(F.nvert + g);
}
// NV0: the block's nvert is zero everywhere (no immersed body), known on the
// host, so every nvert test folds away at compile time
template <bool NV0, class RG>
__device__ __forceinline__ double nvert_v(const DevCfg &c, const DevFields &F, const RG &Rg, NRef n, long long g) {
  return NV0 ? 0.0 : nvert_at(c, F, Rg, n, g);
}
// the same for a node that may lie beyond the ring's i/j halo
template <bool NV0, class RG>
__device__ __forceinline__ double nvert_far(const DevCfg &c, const DevFields &F, const RG &Rg, NRef n, long long g) {
  if (NV0) return 0.0;
  return (c.nvq && Rg.holds(n)) ? Rg.nv(n) : ldg(F.nvert + g);
}

// ---------------------------------------------------------------- recon --
// minmod (rhs.c:2256-2307): 0 where a and b have opposite signs, else
// sgn(a) * min(|a|, |b|), formed here branch-free as the smaller magnitude
// with the sign of a -- the same value (a zero slope may come out as -0,
// which the MUSCL sum q0 +- 0.5 * slope absorbs)
template <typename R>
__device__ __forceinline__ R r_minmod(R a, R b) {
  const R m = copysign(fmin(fabs(a), fabs(b)), a);
  return (a * b < R(0)) ? R(0.) : m;
}
template <typename R>
__device__ __forceinline__ R muscl_l(R qm, R q0, R qp) { return q0 + R(0.5) * r_minmod(qp - q0, q0 - qm); }
template <typename R>
__device__ __forceinline__ R muscl_r(R qm, R q0, R qp) { return q0 - R(0.5) * r_minmod(qp - q0, q0 - qm); }
template <typename R>
__device__ __forceinline__ R weno3_l(R qm, R q0, R qp) {
  const R d0 = R(0.6666667), d1 = R(0.3333333), eps = R(1e-6);  // rhs.c:2386 (truncated weights)
  R r0 = R(0.5) * q0 + R(0.5) * qp, r1 = R(-0.5) * qm + R(1.5) * q0;
  R b0 = (qp - q0) * (qp - q0), b1 = (qm - q0) * (qm - q0);
  R a0 = d0 / ((eps + b0) * (eps + b0)), a1 = d1 / ((eps + b1) * (eps + b1));
  R as = a0 + a1;
  return (a0 / as) * r0 + (a1 / as) * r1;
}
template <typename R>
__device__ __forceinline__ R weno3_r(R qm, R q0, R qp) {
  const R d0 = R(0.6666667), d1 = R(0.3333333), eps = R(1e-6);
  R r0 = R(1.5) * q0 - R(0.5) * qp, r1 = R(0.5) * qm + R(0.5) * q0;
  R b0 = (qp - q0) * (qp - q0), b1 = (qm - q0) * (qm - q0);
  R a0 = d0 / ((eps + b0) * (eps + b0)), a1 = d1 / ((eps + b1) * (eps + b1));
  R as = a0 + a1;
  return (a0 / as) * r0 + (a1 / as) * r1;
}
template <typename R>
__device__ __forceinline__ R eno_r(R qm, R q0, R qp, int k) {
  if (k == 2) return R(0.5) * q0 + R(0.5) * qp;
  return -qm * R(0.1666666666666666) + q0 * R(0.8333333333333333) + qp * R(0.3333333333333333);
}
template <typename R>
__device__ __forceinline__ R eno_l(R qm, R q0, R qp, int k) {
  if (k == 2) return R(0.5) * q0 + R(0.5) * qm;
  return qm * R(0.3333333333333333) + q0 * R(0.8333333333333333) - qp * R(0.1666666666666666);
}

// WENO5-JS (Jiang & Shu, J. Comput. Phys. 126 (1996) 202-228; no counterpart
// in the reference): value at x_{i+1/2} from a..e = v_{i-2..i+2}, left-biased;
// candidates q_k (times 6), smoothness beta_k = 13/12 (2nd difference)^2 +
// 1/4 (slope)^2, weights d_k / (eps + beta_k)^2 with d = (0.1, 0.6, 0.3) and
// eps = 1e-6, value sum(alpha_k q_k) / (6 sum(alpha_k)).  The right-biased
// value at x_{i+1/2} is weno5(v_{i+3}, .., v_{i-1}).  Same operation order as
// the oracle's restatement (bit-identical in the FP64 form).
template <typename R>
__device__ __forceinline__ R weno5(R a, R b, R c, R d, R e) {
  const R eps = R(1e-6), c13 = R(13.0 / 12.0);
  const R q0 = (R(2.0) * a - R(7.0) * b) + R(11.0) * c;
  const R q1 = (R(5.0) * c - b) + R(2.0) * d;
  const R q2 = (R(2.0) * c + R(5.0) * d) - e;
  const R t0 = (a - R(2.0) * b) + c, u0 = (a - R(4.0) * b) + R(3.0) * c;
  const R t1 = (b - R(2.0) * c) + d, u1 = b - d;
  const R t2 = (c - R(2.0) * d) + e, u2 = (R(3.0) * c - R(4.0) * d) + e;
  const R b0 = c13 * (t0 * t0) + R(0.25) * (u0 * u0);
  const R b1 = c13 * (t1 * t1) + R(0.25) * (u1 * u1);
  const R b2 = c13 * (t2 * t2) + R(0.25) * (u2 * u2);
  const R a0 = R(0.1) / ((eps + b0) * (eps + b0));
  const R a1 = R(0.6) / ((eps + b1) * (eps + b1));
  const R a2 = R(0.3) / ((eps + b2) * (eps + b2));
  return ((a0 * q0 + a1 * q1) + a2 * q2) / (R(6.0) * ((a0 + a1) + a2));
}

// Conserved state and pressure of one node as the ring stores them, from its
// raw FP64 state v (EqOfState rhs.c:4850; the mixed form shifts by the
// reference state); pst/pin: the carried pressure of the FP64 form.  The
// ring's derive pass and the global-memory path of far stencil nodes share
// this arithmetic.
template <typename R, bool MIX>
__device__ __forceinline__ void node_qp(const DevCfg &c, const double v[5], bool pst, double pin, R q[5], R &p) {
  double pp = 0.0, e = v[4];
  if (v[0] != 0.0) {
    if (MIX) {
      const double ri = 1.0 / v[0];
      pp = (c.gamma - 1) * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) * ri);
      e -= c.e_ref;
      pp -= c.p_ref;
    } else {
      pp = pst ? pin : (c.gamma - 1) * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0]);
    }
  }
#pragma unroll
  for (int a = 0; a < 4; a++) q[a] = R(v[a]);
  q[4] = R(e);
  p = R(pp);
}

// Rusanov flux on reconstructed states (rhs.c:2769-2810), same operation
// order as the reference (divisions, no reciprocal reuse).  In the mixed form
// pL/pR are p - p_ref (the sound speed adds p_ref back) and Uf returns the
// face velocity measure 0.5*(uconL + uconR) that multiplies H_ref.
// The mixed form multiplies by one reciprocal of each state's density
// instead of dividing by it four times (FP32 rounding differences only).
template <typename R, bool MIX>
__device__ __forceinline__ void rusanov(const R QL[5], const R QR[5], R pL, R pR, const R h[3], bool use_qr_for_l,
                                        bool r_from_l, R pref, R F[5], R &Uf) {
  R uconL, uconR, cL, cR;
  if constexpr (MIX) {
    const R ril = R(1) / QL[0], rir = R(1) / QR[0];
    const R UR = (h[0] * QR[1] + h[1] * QR[2] + h[2] * QR[3]) * rir;
    uconL = use_qr_for_l ? UR : (h[0] * QL[1] + h[1] * QL[2] + h[2] * QL[3]) * ril;
    uconR = r_from_l ? uconL : UR;
    cL = R(GAMMA_CONV) * (pL + pref) * ril;
    cR = R(GAMMA_CONV) * (pR + pref) * rir;
  } else {
    uconL = use_qr_for_l ? (h[0] * (QR[1] / QR[0]) + h[1] * (QR[2] / QR[0]) + h[2] * (QR[3] / QR[0]))
                         : (h[0] * (QL[1] / QL[0]) + h[1] * (QL[2] / QL[0]) + h[2] * (QL[3] / QL[0]));
    uconR = r_from_l ? uconL : (h[0] * (QR[1] / QR[0]) + h[1] * (QR[2] / QR[0]) + h[2] * (QR[3] / QR[0]));
    cL = R(GAMMA_CONV) * pL / QL[0];
    cR = R(GAMMA_CONV) * pR / QR[0];
  }
  R gii = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
  R saL = fabs(uconL) + sqrt(fabs(cL) * gii);
  R saR = fabs(uconR) + sqrt(fabs(cR) * gii);
  R SA = (saL < saR) ? saR : saL;
  F[0] = R(0.5) * (QL[0] * uconL + QR[0] * uconR) - R(0.5) * SA * (QR[0] - QL[0]);
#pragma unroll
  for (int a = 0; a < 3; a++)
    F[1 + a] = R(0.5) * ((QL[1 + a] * uconL + QR[1 + a] * uconR) + (pL * h[a] + pR * h[a])) - R(0.5) * SA * (QR[1 + a] - QL[1 + a]);
  F[4] = R(0.5) * ((pL + QL[4]) * uconL + (pR + QR[4]) * uconR) - R(0.5) * SA * (QR[4] - QL[4]);
  Uf = MIX ? R(0.5) * (uconL + uconR) : R(0);
}

// Roe's approximate Riemann solver with Harten's entropy fix (no counterpart
// in the reference; Roe, J. Comput. Phys. 43 (1981); Harten, J. Comput.
// Phys. 49 (1983)): the central part is the Rusanov flux's average of the
// two physical fluxes; the dissipation is |h| |A~| (QR - QL) of the
// Roe-averaged Jacobian along n = h/|h|, acoustic speeds below 0.1 c~
// smoothed to (l^2 + delta^2) / (2 delta).  Mixed form: the enthalpy adds
// back H_ref; pressure and energy differences are shift-free.
template <typename R, bool MIX>
__device__ __forceinline__ void roe(const R QL[5], const R QR[5], R pL, R pR, const R h[3], bool use_qr_for_l,
                                    bool r_from_l, R pref, R href, R F[5], R &Uf) {
  (void)pref;
  const R g = R(GAMMA_CONV);
  // the mixed form multiplies by reciprocals of the densities, the face area
  // and the root sum (FP32 rounding differences only)
  const R ril = MIX ? R(1) / QL[0] : R(0), rir = MIX ? R(1) / QR[0] : R(0);
#define CB_DIVL(x) (MIX ? (x) * ril : (x) / QL[0])
#define CB_DIVR(x) (MIX ? (x) * rir : (x) / QR[0])
  R uconL = use_qr_for_l ? (h[0] * CB_DIVR(QR[1]) + h[1] * CB_DIVR(QR[2]) + h[2] * CB_DIVR(QR[3]))
                         : (h[0] * CB_DIVL(QL[1]) + h[1] * CB_DIVL(QL[2]) + h[2] * CB_DIVL(QL[3]));
  R uconR = r_from_l ? uconL : (h[0] * CB_DIVR(QR[1]) + h[1] * CB_DIVR(QR[2]) + h[2] * CB_DIVR(QR[3]));
  const R area = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
  const R ria = MIX ? R(1) / area : R(0);
  const R nx = MIX ? h[0] * ria : h[0] / area, ny = MIX ? h[1] * ria : h[1] / area, nz = MIX ? h[2] * ria : h[2] / area;
  const R sl = sqrt(QL[0]), sr = sqrt(QR[0]);
  const R ris = MIX ? R(1) / (sl + sr) : R(0);
  const R wl = MIX ? sl * ris : sl / (sl + sr), wr = MIX ? sr * ris : sr / (sl + sr);
  const R uL = CB_DIVL(QL[1]), vL = CB_DIVL(QL[2]), zL = CB_DIVL(QL[3]);
  const R uR = CB_DIVR(QR[1]), vR = CB_DIVR(QR[2]), zR = CB_DIVR(QR[3]);
  const R HL = CB_DIVL(MIX ? (QL[4] + pL + href) : (QL[4] + pL));
  const R HR = CB_DIVR(MIX ? (QR[4] + pR + href) : (QR[4] + pR));
#undef CB_DIVL
#undef CB_DIVR
  const R rt = sl * sr, ut = wl * uL + wr * uR, vt = wl * vL + wr * vR, zt = wl * zL + wr * zR;
  const R Ht = wl * HL + wr * HR, q2 = ut * ut + vt * vt + zt * zt;
  const R c2 = (g - R(1.0)) * (Ht - R(0.5) * q2), ct = sqrt(fabs(c2));
  const R Unt = ut * nx + vt * ny + zt * nz;
  const R dp = pR - pL, dr = QR[0] - QL[0];
  const R du = uR - uL, dv = vR - vL, dz = zR - zL, dUn = du * nx + dv * ny + dz * nz;
  const R a1 = (dp - rt * ct * dUn) / (R(2.0) * c2), a2 = dr - dp / c2, a3 = (dp + rt * ct * dUn) / (R(2.0) * c2);
  R l1 = fabs(Unt - ct), l2 = fabs(Unt), l3 = fabs(Unt + ct);
  const R delta = R(0.1) * ct;
  if (l1 < delta) l1 = (l1 * l1 + delta * delta) / (R(2.0) * delta);
  if (l3 < delta) l3 = (l3 * l3 + delta * delta) / (R(2.0) * delta);
  const R s1 = l1 * a1, s2 = l2 * a2, s3 = l3 * a3, ss = l2 * rt;
  R D[5];
  D[0] = s1 + s2 + s3;
  D[1] = s1 * (ut - ct * nx) + s2 * ut + s3 * (ut + ct * nx) + ss * (du - dUn * nx);
  D[2] = s1 * (vt - ct * ny) + s2 * vt + s3 * (vt + ct * ny) + ss * (dv - dUn * ny);
  D[3] = s1 * (zt - ct * nz) + s2 * zt + s3 * (zt + ct * nz) + ss * (dz - dUn * nz);
  D[4] = s1 * (Ht - Unt * ct) + s2 * R(0.5) * q2 + s3 * (Ht + Unt * ct) + ss * (ut * du + vt * dv + zt * dz - Unt * dUn);
  F[0] = R(0.5) * (QL[0] * uconL + QR[0] * uconR) - R(0.5) * area * D[0];
#pragma unroll
  for (int a = 0; a < 3; a++)
    F[1 + a] = R(0.5) * ((QL[1 + a] * uconL + QR[1 + a] * uconR) + (pL * h[a] + pR * h[a])) - R(0.5) * area * D[1 + a];
  F[4] = R(0.5) * ((pL + QL[4]) * uconL + (pR + QR[4]) * uconR) - R(0.5) * area * D[4];
  Uf = MIX ? R(0.5) * (uconL + uconR) : R(0);
}

// ------------------------------------------------------- inviscid face ----
// WENO5-JS states of the face pos+1/2 along d (node a at stencil offset 0);
// Q/P hold offsets -1 .. 2 from the ring.  Returns false, leaving the states
// alone, where the stencil pos-2 .. pos+3 leaves the nodes 0 .. m-1 or holds
// a wall node (nvert > 2.9).  Offsets -2 and +3 come from the ring when it
// holds them (always along k) and otherwise from global memory through the
// ring's own node arithmetic.
template <typename R, bool MIX, bool NV0, class RG>
__device__ __forceinline__ bool weno5_face(const DevCfg &c, const DevFields &F, const RG &Rg, NRef a, int d, int pos,
                                           int m, long long g0, long long sd, const R Q[4][5], const R P[4], R QL[5],
                                           R QR[5], R &pL, R &pR) {
  if (pos < 2 || pos > m - 4) return false;
  const NRef nm2 = nshift(a, d, -2), np3 = nshift(a, d, 3);
  if (!NV0) {
    if (nvert_far<NV0>(c, F, Rg, nm2, g0 - 2 * sd) > BLANKWALL || nvert_v<NV0>(c, F, Rg, nshift(a, d, -1), g0 - sd) > BLANKWALL ||
        nvert_v<NV0>(c, F, Rg, nshift(a, d, 2), g0 + 2 * sd) > BLANKWALL ||
        nvert_far<NV0>(c, F, Rg, np3, g0 + 3 * sd) > BLANKWALL)
      return false;
  }
  R Qm[5], Pm, Qp[5], Pp;
  const bool pst = !MIX && F.pin != nullptr;
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const NRef n = t ? np3 : nm2;
    R *qd = t ? Qp : Qm;
    R &pd = t ? Pp : Pm;
    if (d == 2 || Rg.holds(n)) {
#pragma unroll
      for (int q = 0; q < 5; q++) qd[q] = Rg.get(F_RHO + q, n);
      pd = Rg.get(F_P, n);
    } else {
      const long long g = g0 + (t ? 3 : -2) * sd;
      double v[5];
#pragma unroll
      for (int q = 0; q < 5; q++) v[q] = ldg(F.q[q] + g);
      node_qp<R, MIX>(c, v, pst, pst ? ldg(F.pin + g) : 0.0, qd, pd);
    }
  }
#pragma unroll
  for (int q = 0; q < 5; q++) {
    QL[q] = weno5(Qm[q], Q[0][q], Q[1][q], Q[2][q], Q[3][q]);
    QR[q] = weno5(Qp[q], Q[3][q], Q[2][q], Q[1][q], Q[0][q]);
  }
  pL = weno5(Pm, P[0], P[1], P[2], P[3]);
  pR = weno5(Pp, P[3], P[2], P[1], P[0]);
  return true;
}

// Face between node A (tile ref a, global (gi,gj,gk)) and A + e_d.
// DIR >= 0: the face direction as a compile-time constant, so every stencil
// shift, stride and metric selection folds into fixed offsets; DIR = -1: the
// direction is the runtime argument drt (one copy of the code for all three).
// FLUX bits: FLUX_ROE selects Roe's flux instead of Rusanov's.  With the
// sensor off the LES blend weight is the option value s_x = s_y = s_z on
// every face; the host sets FLUX_SIGMA1 when it is 1 and FLUX_SIGMA0 when it
// is 0, and the face then skips the part the blend multiplies by exactly
// zero: (1 - 1) * Fw + 1 * Fc = Fc and (1 - 0) * Fw + 0 * Fc = Fw for finite
// fluxes (the sign of a zero flux aside), so the result is the reference's.
// FLUX_W5: where the reference would reconstruct by WENO3 (fluxorder 3),
// faces whose six-node stencil pos-2 .. pos+3 lies on the nodes 0 .. m-1 and
// holds no wall node take WENO5-JS; the others keep the reference's path, and
// the (j < 30 && k < 7) MUSCL override of the non-LES scheme is off.
template <typename R, bool MIX, bool LES, class RG, int DIR, int FLUX = 0, bool NV0 = false>
__device__ __forceinline__ void conv_face(const DevCfg &c, const DevFields &F, const RG &Rg, NRef a,
                                          int gi, int gj, int gk, int drt, R Fc[5]) {
  const int d = DIR >= 0 ? DIR : drt;
  const long long g0 = gidx(c, gi, gj, gk), sd = gstride(c, d);
  const int pos = d == 0 ? gi : (d == 1 ? gj : gk);
  const int m = d == 0 ? c.mx : (d == 1 ? c.my : c.mz);
  const double nvm = nvert_v<NV0>(c, F, Rg, nshift(a, d, -1), g0 - sd), nv0 = nvert_v<NV0>(c, F, Rg, a, g0),
               nv1 = nvert_v<NV0>(c, F, Rg, nshift(a, d, 1), g0 + sd),
               nv2 = nvert_v<NV0>(c, F, Rg, nshift(a, d, 2), g0 + 2 * sd);
  constexpr bool SMET = StageMet<MIX, NV0, FLUX>::on;
  MetV<R> m0, m1;
  if constexpr (SMET) {
    static_assert(DIR >= 0, "the metric slot needs the face direction at compile time");
    const float4 a0 = Rg.met(d, a);
    const float4 a1 = d < 2 ? Rg.met(d, nshift(a, d, 1)) : __ldg(F.met4[2] + g0 + sd);  // k-face: plane k+1
    m0 = MetV<R>{R(a0.x), R(a0.y), R(a0.z), R(a0.w)};
    m1 = MetV<R>{R(a1.x), R(a1.y), R(a1.z), R(a1.w)};
  } else {
    m0 = met_load<R, MIX>(F, d, g0);
    m1 = met_load<R, MIX>(F, d, g0 + sd);
  }
  R h[3];
  h[0] = R(0.5) * (m0.x + m1.x);
  h[1] = R(0.5) * (m0.y + m1.y);
  h[2] = R(0.5) * (m0.z + m1.z);
  const R pref = R(c.p_ref), href = R(c.h_ref);

  // stencil values along d: s=0..3 -> node offsets -1..2
  R Q[4][5], P[4];
#pragma unroll
  for (int s = 0; s < 4; s++) {
    NRef n = nshift(a, d, s - 1);
#pragma unroll
    for (int q = 0; q < 5; q++) Q[s][q] = Rg.get(F_RHO + q, n);
    P[s] = Rg.get(F_P, n);
  }

  constexpr bool ROE = (FLUX & FLUX_ROE) != 0;
  constexpr bool W5 = (FLUX & FLUX_W5) != 0;
  constexpr bool CEN_ONLY = LES && (FLUX & FLUX_SIGMA1) != 0;
  constexpr bool UPW_ONLY = LES && (FLUX & FLUX_SIGMA0) != 0;
  R Fw[5], Ufw = R(0);
#pragma unroll
  for (int q = 0; q < 5; q++) Fw[q] = R(0);
  if constexpr (!CEN_ONLY) {  // reconstruction and the upwind flux
    R QL[5], QR[5], pL, pR;
    constexpr bool PLAIN = (FLUX & FLUX_PLAIN) != 0;
    const int fo = (PLAIN && !W5) ? 2 : c.fluxorder;
    bool first;
    if (LES) {
      double nsum2 = (d == 2) ? nv0 + (NV0 ? 0.0 : ldg(F.nvert + gidx(c, 1, gj, gk + 1))) : nv0 + nv1;  // quirk rhs.c:4046
      first = fo == 1 || (!PLAIN && (pos == 0 || pos == m - 2) && bc_lo(c, d) != 7) || nsum2 > BLANKWALL;
    } else {
      first = fo == 1 || pos == 0 || pos == m - 2 || (nv0 + nv1) > BLANKWALL;
    }
    int iso_case = 0;
    if (!LES && !PLAIN && d == 1 && c.isothermal) {
      if (gj == 0 && c.bctype[2] == 1) iso_case = 1;           // rhs.c:2822
      else if (gj == m - 2 && c.bctype[3] == 1) iso_case = 2;  // rhs.c:2828
    }
    if (iso_case == 1) {
  #pragma unroll
      for (int q = 0; q < 5; q++) QL[q] = QR[q] = Q[1][q];
      pL = pR = P[1];
    } else if (iso_case == 2) {
  #pragma unroll
      for (int q = 0; q < 5; q++) QL[q] = QR[q] = Q[2][q];
      pL = pR = P[2];
    } else if (first) {
  #pragma unroll
      for (int q = 0; q < 5; q++) { QL[q] = Q[1][q]; QR[q] = Q[2][q]; }
      pL = P[1]; pR = P[2];
    } else if (fo == 2 || (!LES && !W5 && d > 0 && gj < 30 && gk < 7)) {  // quirk rhs.c:2840, 2997
      const bool wm = nvm > BLANKWALL;  // qm = q[i+1] when i-1 is a wall
      const bool wp = nv2 > BLANKWALL;  // qp = q[i] when i+2 is a wall
  #pragma unroll
      for (int q = 0; q < 5; q++) {
        QL[q] = muscl_l(wm ? Q[2][q] : Q[0][q], Q[1][q], Q[2][q]);
        QR[q] = muscl_r(Q[1][q], Q[2][q], wp ? Q[1][q] : Q[3][q]);
      }
      pL = muscl_l(wm ? P[2] : P[0], P[1], P[2]);
      pR = muscl_r(P[1], P[2], wp ? P[1] : P[3]);
    } else if (W5 && weno5_face<R, MIX, NV0>(c, F, Rg, a, d, pos, m, g0, sd, Q, P, QL, QR, pL, pR)) {
      // WENO5-JS reconstruction of Q and p
    } else {
      const int ord = c.eno_order;
      const bool el = nvm > BLANKWALL && (d != 0 || (gi + 2) < c.mx);
      const bool er = nv2 > BLANKWALL;
      if (el) {
  #pragma unroll
        for (int q = 0; q < 5; q++) QL[q] = eno_l(Q[1][q], Q[2][q], Q[3][q], ord);
        pL = eno_l(P[1], P[2], P[3], ord);
      } else {
  #pragma unroll
        for (int q = 0; q < 5; q++) QL[q] = weno3_l(Q[0][q], Q[1][q], Q[2][q]);
        pL = weno3_l(P[0], P[1], P[2]);
        if (!LES && !PLAIN && d == 1 && gj == 1 && c.isothermal && c.bctype[2] == 1) {  // rhs.c:2926
          QL[0] = eno_l(Q[1][0], Q[2][0], Q[3][0], ord);
          QL[4] = eno_l(Q[1][4], Q[2][4], Q[3][4], ord);
          pL = eno_l(P[1], P[2], P[3], ord);
        }
      }
      if (er) {
  #pragma unroll
        for (int q = 0; q < 5; q++) QR[q] = eno_r(Q[0][q], Q[1][q], Q[2][q], ord);
        pR = eno_r(P[0], P[1], P[2], ord);
      } else {
  #pragma unroll
        for (int q = 0; q < 5; q++) QR[q] = weno3_r(Q[1][q], Q[2][q], Q[3][q]);
        pR = weno3_r(P[1], P[2], P[3]);
      }
    }
    if (LES) {
      if (ROE) roe<R, MIX>(QL, QR, pL, pR, h, false, false, pref, href, Fw, Ufw);
      else rusanov<R, MIX>(QL, QR, pL, pR, h, false, false, pref, Fw, Ufw);
    } else {
      const bool use_qr_l = !PLAIN && (pos == m - 2 && bc_hi(c, d) == 1);
      const bool r_from_l = !PLAIN && (pos == 0 && bc_lo(c, d) == 1);
      if (ROE) roe<R, MIX>(QL, QR, pL, pR, h, use_qr_l, r_from_l, pref, href, Fw, Ufw);
      else rusanov<R, MIX>(QL, QR, pL, pR, h, use_qr_l, r_from_l, pref, Fw, Ufw);
    }
  }
  if (!LES) {
#pragma unroll
    for (int q = 0; q < 5; q++) Fc[q] = Fw[q];
    if (MIX) Fc[4] += href * Ufw;
    return;
  }

  if constexpr (UPW_ONLY) {
#pragma unroll
    for (int q = 0; q < 5; q++) Fc[q] = Fw[q];
    if (MIX) Fc[4] += href * Ufw;
    return;
  }
  // central flux (rhs.c:3483-3547) and blend
  R Fcen[5], Ufc;
  bool four = false;
  if (pos > 0 && pos < m - 2) {
    double nsum = (d == 0) ? nv0 + nv1 + nv2 + nvm : nvm + nv0 + nv1 + nv2;
    four = nsum < 2.9;
  }
  if (four && (c.central == 2 || c.central == 3)) {
    R U[4], EP[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const MetV<R> ms = s == 1 ? m0 : (s == 2 ? m1 : met_load<R, MIX>(F, d, g0 + (s - 1) * sd));
      U[s] = R(1.) / Q[s][0] * (ms.x * Q[s][1] + ms.y * Q[s][2] + ms.z * Q[s][3]);
      EP[s] = P[s] + Q[s][4];
    }
    const R fp4 = R(1.0) / R(12.0) * (-P[0] + R(7) * P[1] + R(7) * P[2] - P[3]);
    if (c.central == 2) {
#define CB_FP2(A0, A1, A2, A3) ((A1 + A2) * (U[1] + U[2]) / R(3.0) - R(1.) / R(24.) * (A0 * U[0] + A0 * U[2] + A1 * U[1] + A1 * U[3] + A2 * U[2] + A2 * U[0] + A3 * U[1] + A3 * U[3]))
      Fcen[0] = CB_FP2(Q[0][0], Q[1][0], Q[2][0], Q[3][0]);
      Fcen[1] = CB_FP2(Q[0][1], Q[1][1], Q[2][1], Q[3][1]) + fp4 * h[0];
      Fcen[2] = CB_FP2(Q[0][2], Q[1][2], Q[2][2], Q[3][2]) + fp4 * h[1];
      Fcen[3] = CB_FP2(Q[0][3], Q[1][3], Q[2][3], Q[3][3]) + fp4 * h[2];
      Fcen[4] = CB_FP2(EP[0], EP[1], EP[2], EP[3]);
      Ufc = MIX ? CB_FP2(R(1), R(1), R(1), R(1)) : R(0);
#undef CB_FP2
    } else {
#define CB_FP1(A0, A1, A2, A3) (R(1.0) / R(12.0) * (-A0 * U[0] + R(7) * A1 * U[1] + R(7) * A2 * U[2] - A3 * U[3]))
      Fcen[0] = CB_FP1(Q[0][0], Q[1][0], Q[2][0], Q[3][0]);
      Fcen[1] = CB_FP1(Q[0][1], Q[1][1], Q[2][1], Q[3][1]) + fp4 * h[0];
      Fcen[2] = CB_FP1(Q[0][2], Q[1][2], Q[2][2], Q[3][2]) + fp4 * h[1];
      Fcen[3] = CB_FP1(Q[0][3], Q[1][3], Q[2][3], Q[3][3]) + fp4 * h[2];
      Fcen[4] = CB_FP1(EP[0], EP[1], EP[2], EP[3]);
      Ufc = MIX ? CB_FP1(R(1), R(1), R(1), R(1)) : R(0);
#undef CB_FP1
    }
  } else {
    const R rc = R(0.5) * (Q[1][0] + Q[2][0]), uc = R(0.5) * (Q[1][1] + Q[2][1]), vc = R(0.5) * (Q[1][2] + Q[2][2]);
    const R wc = R(0.5) * (Q[1][3] + Q[2][3]), ec = R(0.5) * (Q[1][4] + Q[2][4]);
    const R Uc = (h[0] * uc + h[1] * vc + h[2] * wc) / rc;
    const R pa = R(0.5) * (P[1] + P[2]);
    Fcen[0] = rc * Uc;
    Fcen[1] = uc * Uc + pa * h[0];
    Fcen[2] = vc * Uc + pa * h[1];
    Fcen[3] = wc * Uc + pa * h[2];
    Fcen[4] = Uc * (ec + pa);
    Ufc = MIX ? Uc : R(0);
  }
  if constexpr (CEN_ONLY) {
#pragma unroll
    for (int q = 0; q < 5; q++) Fc[q] = Fcen[q];
    if (MIX) Fc[4] += href * Ufc;
    return;
  }
  const R sigma = R(sigma_at(c, F, d, gi, gj, gk));
#pragma unroll
  for (int q = 0; q < 5; q++) Fc[q] = Fw[q] * (R(1.0) - sigma) + Fcen[q] * sigma;
  if (MIX) Fc[4] += href * (Ufw * (R(1.0) - sigma) + Ufc * sigma);
}

// -------------------------------------------------------- viscous face ----
__device__ __forceinline__ bool blocked(double v) { return v > SOLID && v < INNERBLANK; }

// FLUX bits as for conv_face: with the metric slot (StageMet) the metric
// vectors and nu_t of the face's plane-k nodes come from shared memory, and a
// constant blend weight (FLUX_SIGMA0 / FLUX_SIGMA1) is the value the sigma of
// every node takes.  The mixed form groups its FP32 terms for FMA: the
// divergence as the trace of r, one factor aj*nu, the heat-flux constant
// gamma / (Pr (gamma - 1)) from the host.
template <typename R, bool MIX, bool LES, class RG, int DIR, bool NV0 = false, int FLUX = 0>
__device__ __forceinline__ void visc_face(const DevCfg &c, const DevFields &F, const RG &Rg, NRef a,
                                          int gi, int gj, int gk, int drt, R Fv[5], R A[3]) {
  constexpr bool SMET = StageMet<MIX, NV0, FLUX>::on;
  static_assert(!SMET || (MIX && DIR >= 0), "the metric slot holds FP32 vectors, selected at compile time");
  const int d = DIR >= 0 ? DIR : drt;
  const long long g0 = gidx(c, gi, gj, gk), sd = gstride(c, d), g1 = g0 + sd;
  const int pos = d == 0 ? gi : (d == 1 ? gj : gk);
  const int m = d == 0 ? c.mx : (d == 1 ? c.my : c.mz);
  const NRef b = nshift(a, d, 1);
  // D[f][e]: derivative of (u, v, w, T) along computational direction e
  R D[4][3];
#pragma unroll
  for (int e = 0; e < 3; e++) {
    if (e == d) {
#pragma unroll
      for (int f = 0; f < 4; f++) D[f][e] = Rg.get(F_U + f, b) - Rg.get(F_U + f, a);
      continue;
    }
    const long long te = gstride(c, e);
    const NRef ap = nshift(a, e, 1), am = nshift(a, e, -1), bp = nshift(b, e, 1), bm = nshift(b, e, -1);
    const bool plus_blocked =
        blocked(nvert_v<NV0>(c, F, Rg, ap, g0 + te)) || blocked(nvert_v<NV0>(c, F, Rg, bp, g1 + te));
    const bool minus_blocked =
        blocked(nvert_v<NV0>(c, F, Rg, am, g0 - te)) || blocked(nvert_v<NV0>(c, F, Rg, bm, g1 - te));
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const int fi = F_U + f;
      if (plus_blocked) {
        if (f == 3 && d == 0 && e == 2)  // quirk: dpdz typo rhs.c:1544-1545
          D[f][e] = (Rg.get(fi, b) + Rg.get(fi, a) - Rg.get(fi, bm) - Rg.get(fi, a)) * R(0.5);
        else
          D[f][e] = (Rg.get(fi, b) + Rg.get(fi, a) - Rg.get(fi, bm) - Rg.get(fi, am)) * R(0.5);
      } else if (minus_blocked) {
        D[f][e] = (Rg.get(fi, bp) + Rg.get(fi, ap) - Rg.get(fi, b) - Rg.get(fi, a)) * R(0.5);
      } else {
        D[f][e] = (Rg.get(fi, bp) + Rg.get(fi, ap) - Rg.get(fi, bm) - Rg.get(fi, am)) * R(0.25);
      }
    }
  }
  constexpr bool PLAIN = (FLUX & FLUX_PLAIN) != 0;
  if (!PLAIN && c.twod == 1) D[0][0] = D[0][1] = D[0][2] = R(0.);  // lUcat x = 0 (CalcUCat rhs.c:1349)
  const R dudc = D[0][0], dude = D[0][1], dudz = D[0][2];
  const R dvdc = D[1][0], dvde = D[1][1], dvdz = D[1][2];
  const R dwdc = D[2][0], dwde = D[2][1], dwdz = D[2][2];
  const R dpdc = D[3][0], dpde = D[3][1], dpdz = D[3][2];

  R mh[3][3];
  R w0[2], w1[2];  // mixed form: filter width and aj at g0 / g1
#pragma unroll
  for (int e = 0; e < 3; e++) {
    MetV<R> p0, p1;
    if constexpr (SMET) {
      const float4 a0 = Rg.met(e, a);
      const float4 a1 = d < 2 ? Rg.met(e, b) : __ldg((e == 0 ? F.met4[0] : (e == 1 ? F.met4[1] : F.met4[2])) + g1);
      p0 = MetV<R>{R(a0.x), R(a0.y), R(a0.z), R(a0.w)};
      p1 = MetV<R>{R(a1.x), R(a1.y), R(a1.z), R(a1.w)};
    } else {
      p0 = met_load<R, MIX>(F, e, g0);
      p1 = met_load<R, MIX>(F, e, g1);
    }
    mh[e][0] = R(0.5) * (p0.x + p1.x);
    mh[e][1] = R(0.5) * (p0.y + p1.y);
    mh[e][2] = R(0.5) * (p0.z + p1.z);
    if (e < 2) { w0[e] = p0.w; w1[e] = p1.w; }
  }
  const R md0 = d == 0 ? mh[0][0] : (d == 1 ? mh[1][0] : mh[2][0]);
  const R md1 = d == 0 ? mh[0][1] : (d == 1 ? mh[1][1] : mh[2][1]);
  const R md2 = d == 0 ? mh[0][2] : (d == 1 ? mh[1][2] : mh[2][2]);
  const R csi0 = mh[0][0], csi1 = mh[0][1], csi2 = mh[0][2];
  const R eta0 = mh[1][0], eta1 = mh[1][1], eta2 = mh[1][2];
  const R zet0 = mh[2][0], zet1 = mh[2][1], zet2 = mh[2][2];
  const R g11 = csi0 * md0 + csi1 * md1 + csi2 * md2;
  const R g21 = eta0 * md0 + eta1 * md1 + eta2 * md2;
  const R g31 = zet0 * md0 + zet1 * md1 + zet2 * md2;

  const R r11 = dudc * csi0 + dude * eta0 + dudz * zet0;
  const R r21 = dvdc * csi0 + dvde * eta0 + dvdz * zet0;
  const R r31 = dwdc * csi0 + dwde * eta0 + dwdz * zet0;
  const R r12 = dudc * csi1 + dude * eta1 + dudz * zet1;
  const R r22 = dvdc * csi1 + dvde * eta1 + dvdz * zet1;
  const R r32 = dwdc * csi1 + dwde * eta1 + dwdz * zet1;
  const R r13 = dudc * csi2 + dude * eta2 + dudz * zet2;
  const R r23 = dvdc * csi2 + dvde * eta2 + dvdz * zet2;
  const R r33 = dwdc * csi2 + dwde * eta2 + dwdz * zet2;

  const R ajc = MIX ? R(0.5) * (w0[1] + w1[1]) : R(0.5) * (R(ldg(F.aj + g0)) + R(ldg(F.aj + g1)));
  R nu = R(c.inv_ren);  // 1./ren (evaluated once on the host, same value)
  if (LES) {
    // quirk: eta/zeta faces average rho over i and i+1 (rhs.c:1835, 2034)
    const R rhs_rho = (d == 0) ? Rg.get(F_RHO, b) : Rg.get(F_RHO, nshift(a, 0, 1));
    nu = R(c.inv_ren_half) * (Rg.get(F_RHO, a) + rhs_rho);  // (1./ren*0.5)*(...)
  }
  // Sutherland's law on the face temperature (rhs.c:1627-1637, 1837-1846,
  // 2036-2045); the hosts never launch the no-IBM variants with it, which
  // keeps their registers for the common path
  if (!NV0 && c.sutherland) {
    const R psum = MIX ? (Rg.get(F_P, a) + Rg.get(F_P, b)) + R(2.0 * c.p_ref) : Rg.get(F_P, a) + Rg.get(F_P, b);
    const R Tr = R(c.gm2) * psum / (Rg.get(F_RHO, a) + Rg.get(F_RHO, b));
    if (Tr < R(0)) nu = R(c.inv_ren);
    else nu = R(c.sut_k1) / (Tr + R(c.sut_k2)) * (MIX ? Tr * sqrt(Tr) : R(pow((double)Tr, 1.5)));
  }
  const R div = MIX ? R(2. / 3.) * ((r11 + r22) + r33)
                    : R(2.) / R(3.) * (dudc * csi0 + dude * eta0 + dudz * zet0 + dvdc * csi1 + dvde * eta1 +
                                       dvdz * zet1 + dwdc * csi2 + dwde * eta2 + dwdz * zet2);
  const R tu = g11 * dudc + g21 * dude + g31 * dudz + r11 * md0 + r21 * md1 + r31 * md2;
  const R tv = g11 * dvdc + g21 * dvde + g31 * dvdz + r12 * md0 + r22 * md1 + r32 * md2;
  const R tw = g11 * dwdc + g21 * dwde + g31 * dwdz + r13 * md0 + r23 * md1 + r33 * md2;
  // deviatoric stress vectors along the face normal (mixed form)
  const R eu = MIX ? tu - div * md0 : R(0), ev = MIX ? tv - div * md1 : R(0), ew = MIX ? tw - div * md2 : R(0);
  Fv[0] = R(0.);
  if constexpr (MIX) {
    const R s = ajc * nu;
    Fv[1] = eu * s;
    Fv[2] = ev * s;
    Fv[3] = ew * s;
  } else {
    Fv[1] = tu * ajc * (nu);
    Fv[2] = tv * ajc * (nu);
    Fv[3] = tw * ajc * (nu);
    Fv[1] -= div * md0 * ajc * nu;
    Fv[2] -= div * md1 * ajc * nu;
    Fv[3] -= div * md2 * ajc * nu;
  }

  R uh[3];
  if (!PLAIN && pos == 0 && bc_lo(c, d) == 1) {
#pragma unroll
    for (int q = 0; q < 3; q++) uh[q] = Rg.get(F_U + q, a);
  } else if (!PLAIN && pos == m - 2 && bc_hi(c, d) == 1) {
#pragma unroll
    for (int q = 0; q < 3; q++) uh[q] = Rg.get(F_U + q, b);
  } else {
#pragma unroll
    for (int q = 0; q < 3; q++) uh[q] = R(0.5) * (Rg.get(F_U + q, b) + Rg.get(F_U + q, a));
  }
  if (!PLAIN && c.twod == 1) uh[0] = R(0.);
  const R gm = R(c.gamma);
  Fv[4] = (Fv[1] * uh[0] + Fv[2] * uh[1] + Fv[3] * uh[2]) +
          (g11 * dpdc + g21 * dpde + g31 * dpdz) * ajc * (MIX ? nu * R(c.kheat) : gm * nu / R(c.pr) / R(c.gm1));

  A[0] = A[1] = A[2] = R(0.);
  if (LES) {  // rhs.c:1677-1710
    // the node weights: the constant the host chose the variant for, or sigma_at
    constexpr bool S0 = (FLUX & FLUX_SIGMA0) != 0, S1 = (FLUX & FLUX_SIGMA1) != 0;
    const int bi = gi + (d == 0), bj = gj + (d == 1), bk = gk + (d == 2);
    const R sa = S0 ? R(0.) : (S1 ? R(1.) : R(sigma_at(c, F, d, gi, gj, gk)));
    const R sb = S0 ? R(0.) : (S1 ? R(1.) : R(sigma_at(c, F, d, bi, bj, bk)));
    const double nu0 = SMET ? Rg.nut(a) : ldg(F.nut + g0);
    const double nu1 = (SMET && d < 2) ? Rg.nut(b) : ldg(F.nut + g1);
    R nut = R(0.5) * (R(nu0) * sa + R(nu1) * sb);
    const R rho_c = R(0.5) * (Rg.get(F_RHO, a) + Rg.get(F_RHO, b));
    const R sigma_c = R(0.5) * (sa + sb);
    if (!PLAIN && ((bc_lo(c, d) == 1 && pos == 0) || (bc_hi(c, d) == 1 && pos == m - 2))) nut = R(0);
    const R S2 = R(.5) * ((r11 - div) * (r11 - div) + r12 * r12 + r13 * r13 + r21 * r21 + (r22 - div) * (r22 - div) +
                          r23 * r23 + r31 * r31 + r32 * r32 + (r33 - div) * (r33 - div));
    // pow(pow(1/aj, 1/3), 2) of the left node, precomputed once per node
    const R pf = MIX ? w0[0] : R(ldg(F.delta2 + g0));
    if constexpr (MIX) {
      const R sn = ajc * (nut * rho_c);
      const R ks = -S2 * pf * R(c.ci * (2.0 / 3.0)) * (rho_c * sigma_c);
      A[0] = eu * sn + ks * md0;
      A[1] = ev * sn + ks * md1;
      A[2] = ew * sn + ks * md2;
    } else {
      const R tx = (tu - div * md0) * ajc * (nut * rho_c);
      const R ty = (tv - div * md1) * ajc * (nut * rho_c);
      const R tz = (tw - div * md2) * ajc * (nut * rho_c);
      const R sgs = -S2 * pf * R(c.ci) * R(2.0) / R(3.0);
      A[0] = tx + sgs * md0 * rho_c * sigma_c;
      A[1] = ty + sgs * md1 * rho_c * sigma_c;
      A[2] = tz + sgs * md2 * rho_c * sigma_c;
    }
    Fv[1] += A[0];
    Fv[2] += A[1];
    Fv[3] += A[2];
  }
}

// Everything one face contributes: the FP64 form keeps conv, visc and the LES
// stress apart (G[0..4], G[5..9], G[10..12]), the mixed form stores visc - conv.
template <typename R, bool MIX, bool LES, bool VISC, class RG, int DIR, int FLUX = 0, bool NV0 = false>
__device__ __forceinline__ void face_flux(const DevCfg &c, const DevFields &F, const RG &Rg, NRef a, int fi,
                                          int fj, int k, int drt, R *G) {
  constexpr int VOFF = FaceWidth<MIX>::VOFF, AOFF = FaceWidth<MIX>::AOFF;
  R Fc[5], Fv[5], A[3];
  conv_face<R, MIX, LES, RG, DIR, FLUX, NV0>(c, F, Rg, a, fi, fj, k, drt, Fc);
  if (VISC) {
    visc_face<R, MIX, LES, RG, DIR, NV0, FLUX>(c, F, Rg, a, fi, fj, k, drt, Fv, A);
  } else {
#pragma unroll
    for (int q = 0; q < 5; q++) Fv[q] = R(0.);
    A[0] = A[1] = A[2] = R(0.);
  }
  if (MIX) {
#pragma unroll
    for (int q = 0; q < 5; q++) G[q] = Fv[q] - Fc[q];
  } else {
#pragma unroll
    for (int q = 0; q < 5; q++) { G[q] = Fc[q]; G[VOFF + q] = Fv[q]; }
  }
  G[AOFF] = A[0]; G[AOFF + 1] = A[1]; G[AOFF + 2] = A[2];
}

// The inviscid half (G[0..4]) or the viscous and SGS half (G[VOFF..VOFF+4],
// G[AOFF..AOFF+2]) of face_flux, for the FP64 form's two threads per face;
// the same calls, so the same values.
template <typename R, bool MIX, bool LES, bool VISC, class RG, int DIR, int FLUX = 0, bool NV0 = false>
__device__ __forceinline__ void face_flux_half(const DevCfg &c, const DevFields &F, const RG &Rg, NRef a, int fi,
                                               int fj, int k, int drt, int role, R *G) {
  constexpr int VOFF = FaceWidth<MIX>::VOFF, AOFF = FaceWidth<MIX>::AOFF;
  static_assert(!MIX, "the mixed form stores visc - conv per face");
  if (role == 0) {
    conv_face<R, MIX, LES, RG, DIR, FLUX, NV0>(c, F, Rg, a, fi, fj, k, drt, G);
  } else {
    R Fv[5], A[3];
    if (VISC) {
      visc_face<R, MIX, LES, RG, DIR, NV0, FLUX>(c, F, Rg, a, fi, fj, k, drt, Fv, A);
    } else {
#pragma unroll
      for (int q = 0; q < 5; q++) Fv[q] = R(0.);
      A[0] = A[1] = A[2] = R(0.);
    }
#pragma unroll
    for (int q = 0; q < 5; q++) G[VOFF + q] = Fv[q];
    G[AOFF] = A[0]; G[AOFF + 1] = A[1]; G[AOFF + 2] = A[2];
  }
}

// ---------------------------------------------------------- the kernel ----
// Tile of 32 x BY interior nodes, NT = 32 (BY + 1) threads (StageGeo).  Per
// plane the block computes 33*BY i-faces, 32*(BY+1) j-faces and 32*BY k-faces
// in three warp-uniform rounds: virtual face v = round*NT + tid maps to
// [0,NT) i-faces, [NT,2NT) j-faces, [2NT,3NT) k-faces, so every warp runs one
// face direction per round (no divergence between directions).
constexpr int SBX = 32, SBY = StageGeo<0>::BY, SNT = StageGeo<0>::NT;  // the WENO3/MUSCL tile: 32 x 7, 256 threads
constexpr int SBY_W5 = StageGeo<FLUX_W5>::BY, SNT_W5 = StageGeo<FLUX_W5>::NT;  // WENO5: 32 x 5, 192 threads
template <typename R, bool MIX, bool NV0 = false, bool W5 = false>
struct StageSmem {
  using G = StageGeo<W5 ? FLUX_W5 : 0>;
  static constexpr int NG = FaceWidth<MIX>::NG;
  static constexpr int PN = G::Tile::PN;
  // FP64 staging fields per plane: 5 state fields, nvert (not with NV0), and
  // in the FP64 form the pressure carried from an immersed step's
  // interpolation (the mixed form keeps that shared memory as L1: the carried
  // value differs from the EOS by <= 1e-12, inside its bar)
  static constexpr int NSTG = 5 + (NV0 ? 0 : 1) + (MIX ? 0 : 1);
  // the metric / nu_t slot of the current plane (StageMet): [3][MPN] float4
  // and [MPN] double
  static constexpr bool SMET = StageMet<MIX, NV0, W5 ? FLUX_W5 : 0>::on;
  static constexpr int MPN = (G::BX + 2) * (G::BY + 2);
  static constexpr size_t MET_BYTES = SMET ? (size_t)MPN * (3 * sizeof(float4) + sizeof(double)) : 0;
  // FP64 staging of the next plane, metric slot, ring, face buffers (with the
  // metric slot the k-faces stay in registers: the thread that forms a k-face
  // is the thread that updates its node), nvert byte ring [NPL][PN] (not with
  // NV0: the no-IBM variants leave that memory to the L1)
  static constexpr size_t bytes =
      sizeof(double) * (size_t)NSTG * PN + MET_BYTES +
      sizeof(R) * ((size_t)G::NPL * NF * PN + (size_t)NG * (G::NXF + G::NYF + (SMET ? 0 : G::NZF))) +
      (NV0 ? 0 : (size_t)G::NPL * PN);
  static_assert((sizeof(double) * NSTG * PN) % 16 == 0, "the metric slot takes 16-byte copies");
};
constexpr size_t STAGE_SMEM_BYTES = StageSmem<double, false>::bytes;
constexpr size_t STAGE_SMEM_BYTES_MIXED = StageSmem<float, true>::bytes;
// dynamic shared memory of a stage-kernel launch
template <typename R, bool MIX, bool NV0, bool W5 = false>
constexpr size_t stage_smem() { return StageSmem<R, MIX, NV0, W5>::bytes; }
static_assert(STAGE_SMEM_BYTES <= 232448, "shared memory budget of one block");
static_assert(StageSmem<double, false, false, true>::bytes <= 232448, "WENO5 FP64: shared memory of one block");
static_assert(2 * (STAGE_SMEM_BYTES_MIXED + 1024) <= 233472, "mixed form: two blocks per SM");
static_assert(2 * (StageSmem<float, true, false, true>::bytes + 1024) <= 233472, "WENO5 mixed: two blocks per SM");
static_assert(2 * (StageSmem<float, true, true, false>::bytes + 1024) <= 233472, "mixed with the metric slot: two blocks per SM");

// All face fluxes of plane k of a tile into the face buffers (ZONLY: just the
// k-faces, for the prologue).  A function rather than a lambda so that it is
// always inlined: an outlined call would copy the kernel parameters to local
// memory.
// With the metric slot (StageMet) the k-face comes back in gzr (registers:
// thread u of the k round is the thread that updates node u); otherwise it
// goes to gzb (the FP64 form forms the two halves of a face in two threads).
template <typename R, bool MIX, bool LES, bool VISC, bool ZONLY, int FLUX, bool NV0, class RG>
__device__ __forceinline__ void plane_faces(const DevCfg &c, const DevFields &F, const RG &Rg, int i0, int j0, int k,
                                            R *gxb, R *gyb, R *gzb, R *gzr) {
  using G = StageGeo<FLUX>;
  constexpr int BX = G::BX, NT = G::NT, NG = FaceWidth<MIX>::NG;
  constexpr bool SPLIT = StageThreads<FLUX, MIX>::SPLIT;
  constexpr int VOFF = FaceWidth<MIX>::VOFF;
  const int tid = threadIdx.x;
  // role 0: the faces' inviscid fluxes; role 1 (FP64 form): their viscous
  // and SGS fluxes (warp-uniform: NT is a multiple of 32)
  const int role = SPLIT ? tid / NT : 0;
#pragma unroll 1
  for (int r = ZONLY ? 2 : 0; r < 3; r++) {
    const int u = SPLIT ? tid - role * NT : tid;  // face index within this round's direction
    int d, fi, fj;
    NRef a;
    R *dst;
    int nslot;
    if (r == 0) {
      d = 0;
      if (u >= G::NXF) continue;
      const int fx = u % (BX + 1), fy = u / (BX + 1);
      fi = i0 - 1 + fx; fj = j0 + fy;
      a = NRef{0, fy + 2, fx + 1};
      dst = gxb; nslot = G::NXF;
    } else if (r == 1) {
      d = 1;
      if (u >= G::NYF) continue;
      const int fx = u % BX, fy = u / BX;
      fi = i0 + fx; fj = j0 - 1 + fy;
      a = NRef{0, fy + 1, fx + 2};
      dst = gyb; nslot = G::NYF;
    } else {
      d = 2;
      if (u >= G::NZF) continue;
      const int fx = u % BX, fy = u / BX;
      fi = i0 + fx; fj = j0 + fy;
      a = NRef{0, fy + 2, fx + 2};
      dst = gzb; nslot = G::NZF;
    }
    R Gf[NG];
    // -twoD 1 forms no i-face flux (rhs.c:1487, 2646, 3465): it stays zero
    const bool live = fi <= c.mx - 2 && fj <= c.my - 2 && !(d == 0 && (FLUX & FLUX_PLAIN) == 0 && c.twod == 1);
    if constexpr (SPLIT) {
      // this thread's half of the face: G[0..4], or G[VOFF..NG-1]
      const int q0 = role == 0 ? 0 : VOFF, q1 = role == 0 ? VOFF : NG;
      if (live) {
        // one instantiation per direction (d is warp-uniform): the index
        // arithmetic of every stencil shift folds into constants (4 % faster
        // than one copy for all directions at 128 registers); the WENO5-JS
        // variants, at 168 registers, keep one copy (13 % faster there)
        if constexpr ((FLUX & FLUX_W5) != 0)
          face_flux_half<R, MIX, LES, VISC, RG, -1, FLUX, NV0>(c, F, Rg, a, fi, fj, k, d, role, Gf);
        else if (d == 0) face_flux_half<R, MIX, LES, VISC, RG, 0, FLUX, NV0>(c, F, Rg, a, fi, fj, k, d, role, Gf);
        else if (d == 1) face_flux_half<R, MIX, LES, VISC, RG, 1, FLUX, NV0>(c, F, Rg, a, fi, fj, k, d, role, Gf);
        else face_flux_half<R, MIX, LES, VISC, RG, 2, FLUX, NV0>(c, F, Rg, a, fi, fj, k, d, role, Gf);
      } else {
#pragma unroll
        for (int q = 0; q < NG; q++) Gf[q] = R(0.);
      }
#pragma unroll
      for (int q = 0; q < NG; q++)
        if (q >= q0 && q < q1) dst[(size_t)q * nslot + u] = Gf[q];
      continue;
    }
    if (live) {
      if constexpr (MIX) {
        // one instantiation per direction (d is warp-uniform): 16 % faster
        // for the FP32 arithmetic of the mixed form
        if (d == 0) face_flux<R, MIX, LES, VISC, RG, 0, FLUX, NV0>(c, F, Rg, a, fi, fj, k, d, Gf);
        else if (d == 1) face_flux<R, MIX, LES, VISC, RG, 1, FLUX, NV0>(c, F, Rg, a, fi, fj, k, d, Gf);
        else face_flux<R, MIX, LES, VISC, RG, 2, FLUX, NV0>(c, F, Rg, a, fi, fj, k, d, Gf);
      } else {
        // one copy for all directions: the FP64 form at 255 registers runs
        // 12 % slower with three
        face_flux<R, MIX, LES, VISC, RG, -1, FLUX, NV0>(c, F, Rg, a, fi, fj, k, d, Gf);
      }
    } else {
#pragma unroll
      for (int q = 0; q < NG; q++) Gf[q] = R(0.);
    }
    if (StageMet<MIX, NV0, FLUX>::on && r == 2) {
#pragma unroll
      for (int q = 0; q < NG; q++) gzr[q] = Gf[q];
      continue;
    }
#pragma unroll
    for (int q = 0; q < NG; q++) dst[(size_t)q * nslot + u] = Gf[q];
  }
  (void)NT;
  (void)VOFF;
  (void)gzb;
}


// One tile column (bxi, byi) of one block over the planes kb .. ke-1: the
// whole k march, with its prologue.
template <typename R, bool MIX, bool LES, bool VISC, bool RHS_MODE, int FLUX = 0, bool NV0 = false>
__device__ __forceinline__ void stage_tile(const DevCfg &c, const DevFields &F, int bxi, int byi, int kb, int ke,
                                           int istage, double alfa, double beta, double adt, double *smem_d) {
  using G = StageGeo<FLUX>;
  constexpr int BX = G::BX, BY = G::BY, NPL = G::NPL, H = G::H;
  constexpr int NT = StageThreads<FLUX, MIX>::N;  // threads of the block
  constexpr int PX = G::Tile::PX, PN = G::Tile::PN, NXF = G::NXF, NYF = G::NYF, NZF = G::NZF;
  constexpr int NG = FaceWidth<MIX>::NG, VOFF = FaceWidth<MIX>::VOFF, AOFF = FaceWidth<MIX>::AOFF;
  constexpr int NSTG = StageSmem<R, MIX, NV0, G::W5>::NSTG;
  using RG = Ring<R, BX, BY, NPL>;
  constexpr bool SMET = StageMet<MIX, NV0, FLUX>::on;
  constexpr int MPX = RG::MPX, MPN = RG::MPN;
  constexpr bool PLAIN = (FLUX & FLUX_PLAIN) != 0;
  double *stg = smem_d;  // [NSTG][PN] raw FP64 Q, nvert and carried pressure of the next plane
  float4 *mts = reinterpret_cast<float4 *>(smem_d + (size_t)NSTG * PN);  // [3][MPN] metric slot (SMET)
  double *nts = reinterpret_cast<double *>(mts + (SMET ? 3 * MPN : 0));   // [MPN] nu_t slot (SMET)
  R *smem = reinterpret_cast<R *>(nts + (SMET ? MPN : 0));
  RG Rg;
  Rg.pl = smem;
  Rg.mt = mts;
  Rg.nt = nts;
  R *gxb = smem + (size_t)NPL * NF * PN;  // [NG][NXF]
  R *gyb = gxb + (size_t)NG * NXF;        // [NG][NYF]
  R *gzb = gyb + (size_t)NG * NYF;        // [NG][NZF] (not with the metric slot)
  unsigned char *nvc = reinterpret_cast<unsigned char *>(gzb + (SMET ? 0 : (size_t)NG * NZF));  // [NPL][PN]
  Rg.nvc = nvc;
  // staged fields per plane: Q, then nvert (byte-exact codes), then lP (carried pressure)
  const bool pst = !MIX && F.pin != nullptr;
  const bool nvs = c.nvq && !NV0;
  const int pslot = nvs ? 6 : 5;

  const int tid = threadIdx.x;
  const int i0 = 1 + bxi * BX, j0 = 1 + byi * BY;
  // node updated by this thread (the last warp only loads and computes faces)
  const int utx = tid % BX, uty = tid / BX;
  const int ugi = i0 + utx, ugj = j0 + uty;
  const bool uact = uty < BY && ugi <= c.mx - 2 && ugj <= c.my - 2;

  // async copy of the raw state of plane kk (with its halo) into the staging
  // buffer: node-major, one index computation per node and one 8-byte copy
  // per staged field (consecutive threads take consecutive nodes of a row, so
  // each field's copies stay coalesced)
  // In the FP64 form the threads of the inviscid half issue the copies and
  // those of the viscous half run the derive pass: the viscous face takes
  // longer, and the inviscid threads also run the node update, in the same
  // phase as the derive pass.
  constexpr bool SPLIT = StageThreads<FLUX, MIX>::SPLIT;
  constexpr int HT = SPLIT ? NT / 2 : NT;  // threads of one half
  auto issue_stage = [&](int kk) {
    const bool kok = kk >= -2 && kk <= c.mz + 1;
    for (int idx = tid; idx < PN && tid < HT; idx += HT) {
      const int ly = idx / PX, lx = idx - ly * PX;
      const int xi = i0 - 2 + lx, yj = j0 - 2 + ly;
      const bool ok = kok && xi <= c.mx + 1 && yj <= c.my + 1;
      const long long go = ok ? gidx(c, xi, yj, kk) : 0;  // src-size 0 below: nothing is read
#pragma unroll
      for (int q = 0; q < 5; q++) cp_async8(stg + q * PN + idx, F.q[q] + go, ok);
      if (nvs) cp_async8(stg + 5 * PN + idx, F.nvert + go, ok);
      if (pst) cp_async8(stg + pslot * PN + idx, F.pin + go, ok);
    }
    cp_async_commit();
  };
  // staging -> ring slot s with the derived p, u, v, w, T (EqOfState rhs.c:4850,
  // CalcUCat rhs.c:1349), all in FP64; the mixed form stores shifted FP32 values
  auto derive = [&](int s) {
    for (int idx = SPLIT ? tid - HT : tid; idx < PN && idx >= 0; idx += HT) {
      double v[NF];
#pragma unroll
      for (int q = 0; q < 5; q++) v[q] = stg[q * PN + idx];
      if (v[0] != 0.0) {
        const double r = v[0];
        if (MIX) {
          // one FP64 reciprocal instead of five divisions: the products differ
          // from the quotients by at most an FP64 ulp, far below the FP32
          // rounding of the shifted values stored next
          const double ri = 1.0 / r;
          v[F_P] = (c.gamma - 1) * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) * ri);
          v[F_U] = v[1] * ri;
          v[F_V] = v[2] * ri;
          v[F_W] = v[3] * ri;
          v[F_T] = v[F_P] * ri;
        } else {  // the reference's quotients (EqOfState rhs.c:4850, CalcUCat rhs.c:1349)
          v[F_P] = pst ? stg[pslot * PN + idx]
                       : (c.gamma - 1) * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / r);
          v[F_U] = v[1] / r;
          v[F_V] = v[2] / r;
          v[F_W] = v[3] / r;
          v[F_T] = v[F_P] / r;
        }
        if (MIX) {
          v[F_RE] -= c.e_ref;
          v[F_P] -= c.p_ref;
          v[F_T] -= c.t_ref;
        }
      } else {
#pragma unroll
        for (int q = 5; q < NF; q++) v[q] = 0.0;
      }
      if constexpr (RG::AOS) {
        float2 *base = reinterpret_cast<float2 *>(Rg.pl + ((size_t)s * PN + idx) * NF);
#pragma unroll
        for (int q = 0; q < NF; q += 2) base[q / 2] = make_float2(float(v[q]), float(v[q + 1]));
      } else {
        R *base = Rg.pl + (size_t)s * NF * PN + idx;
#pragma unroll
        for (int q = 0; q < NF; q++) base[(size_t)q * PN] = R(v[q]);
      }
      if (nvs) nvc[s * PN + idx] = (unsigned char)(stg[5 * PN + idx] * 4.0);
    }
  };
  // async copy of plane kk's FP32 metric vectors and nu_t over the slot's
  // node box into the slot (SMET)
  auto issue_met = [&](int kk) {
    if constexpr (SMET) {
      for (int idx = tid; idx < MPN; idx += NT) {
        const int ly = idx / MPX, lx = idx - ly * MPX;
        const int xi = i0 - 1 + lx, yj = j0 - 1 + ly;
        const bool ok = xi <= c.mx + 1 && yj <= c.my + 1;
        const long long go = ok ? gidx(c, xi, yj, kk) : 0;  // src-size 0 below: nothing is read
#pragma unroll
        for (int e = 0; e < 3; e++) cp_async16(mts + e * MPN + idx, F.met4[e] + go, ok);
        if (LES) cp_async8(nts + idx, F.nut + go, ok);
      }
      cp_async_commit();
    }
  };
  auto load_plane_sync = [&](int kk, int s) {
    issue_stage(kk);
    cp_async_wait_all();
    __syncthreads();
    derive(s);
    __syncthreads();
  };

  // prologue: planes kb-1-H .. kb+H in slots 0 .. NPL-1, k-face kb-1/2 (its
  // stencil is exactly those planes), then plane kb+H+1 into slot 0
  Rg.sb = 0;
  issue_met(kb - 1);  // the metric slot holds plane kb-1 for the prologue's k-face
#pragma unroll 1
  for (int t = 0; t < NPL; t++) load_plane_sync(kb - 1 - H + t, t);
  R gzr[NG];  // with the metric slot: k-face k+1/2 of the node this thread updates
  plane_faces<R, MIX, LES, VISC, true, FLUX, NV0>(c, F, Rg, i0, j0, kb - 1, gxb, gyb, gzb, gzr);  // k-face kb-1/2
  __syncthreads();
  R Gzp[NG];  // k-face k-1/2 of the node this thread updates
#pragma unroll
  for (int q = 0; q < NG; q++) Gzp[q] = uact ? (SMET ? gzr[q] : gzb[(size_t)q * NZF + tid]) : R(0.);
  __syncthreads();
  issue_met(kb);
  load_plane_sync(kb + H + 1, 0);
  int base = 1;  // slot of plane k-H

  for (int k = kb; k < ke; k++) {
    Rg.sb = base;
    const bool more = k + 1 < ke;
    if (more) issue_stage(k + H + 2);  // overlaps the face computation
    if constexpr (SMET) {
      // the k-face k+1/2 of this thread's node reads its far node's metric
      // vectors and nu_t (plane k+1) from global memory in the last face
      // round: start those lines toward L1 while the i and j faces run
      const int fx = tid % BX, fy = tid / BX;
      if (tid < NZF && i0 + fx <= c.mx - 2 && j0 + fy <= c.my - 2) {
        const long long g1 = gidx(c, i0 + fx, j0 + fy, k + 1);
#pragma unroll
        for (int e = 0; e < 3; e++) prefetch_l1(F.met4[e] + g1);
        if (LES) prefetch_l1(F.nut + g1);
      }
    }
    if constexpr (MIX) {
      // the node update's global operands of this plane, from DRAM into L2
      // while the faces run
      if (uact) {
        const long long gu = gidx(c, ugi, ugj, k);
        if (!RHS_MODE) {
#pragma unroll
          for (int q = 0; q < 5; q++) prefetch_l2(F.qold[q] + gu);
          if (istage != 0)
#pragma unroll
            for (int q = 0; q < 5; q++) prefetch_l2(F.q[q] + gu);
        }
#pragma unroll
        for (int a = 0; a < 3; a++) prefetch_l2(F.gcl[a] + gu);
        prefetch_l2(F.aj + gu);
      }
    }
    plane_faces<R, MIX, LES, VISC, false, FLUX, NV0>(c, F, Rg, i0, j0, k, gxb, gyb, gzb, gzr);
    // the only plane k-1 value the update needs, read before that slot is refilled
    const NRef n{0, uty + 2, utx + 2};
    const R rho_km1 = (LES && VISC && uact) ? Rg.get(F_RHO, nshift(n, 2, -1)) : R(0.);
    // the update's global operands, issued before the barrier so that their
    // latency overlaps the wait for the other warps' faces
    const long long g = gidx(c, ugi, ugj, k);
    double qo_r[5], qi_r[5], gcl_r[3], aj_r = 0.;
#pragma unroll
    for (int q = 0; q < 5; q++) qo_r[q] = qi_r[q] = 0.;
    gcl_r[0] = gcl_r[1] = gcl_r[2] = 0.;
    if (uact) {
      aj_r = ldg(F.aj + g);
      if (!RHS_MODE) {
#pragma unroll
        for (int q = 0; q < 5; q++) qo_r[q] = ldg(F.qold[q] + g);
      }
      if (MIX) {
        if (!RHS_MODE && istage != 0) {  // the first stage's combine has no Q term
#pragma unroll
          for (int q = 0; q < 5; q++) qi_r[q] = ldg(F.q[q] + g);
        }
#pragma unroll
        for (int a = 0; a < 3; a++) gcl_r[a] = ldg(F.gcl[a] + g);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    // the faces are done with the metric slot: plane k+1's copies land during
    // the derive pass and the update
    if (more) issue_met(k + 1);
    // plane k+H+2 into the slot of plane k-H (the update reads no value of
    // that plane: rho_km1 above), ahead of the update so that the update's
    // global operands have the derive pass to arrive
    if (more) derive(base);

    if (uact) {
      const double nv = nvert_v<NV0>(c, F, Rg, n, g);
      const int fxr = uty * (BX + 1) + utx + 1, fxl = fxr - 1;   // i+1/2, i-1/2
      const int fyu = (uty + 1) * BX + utx, fyd = uty * BX + utx;  // j+1/2, j-1/2
      const int fz = tid;                                          // k+1/2 (k-1/2 in Gzp)
      // flux differences in the reference's order (rhs.c:3159-3205, 2123-2151):
      // ((((F_i - F_i-1) + F_j) - F_j-1) + F_k) - F_k-1
      auto fdiff = [&](int q) {
        return gxb[(size_t)q * NXF + fxr] - gxb[(size_t)q * NXF + fxl] + gyb[(size_t)q * NYF + fyu] -
               gyb[(size_t)q * NYF + fyd] + (SMET ? gzr[q] : gzb[(size_t)q * NZF + fz]) - Gzp[q];
      };
      // LES energy term (rhs.c:2153-2197): u . sum of rho_face * stress differences
      auto les_energy = [&]() -> R {
        const R r0 = Rg.get(F_RHO, n);
        const R rL = (r0 + Rg.get(F_RHO, nshift(n, 0, -1))) * R(0.5), rR = (Rg.get(F_RHO, nshift(n, 0, 1)) + r0) * R(0.5);
        const R rD = (r0 + Rg.get(F_RHO, nshift(n, 1, -1))) * R(0.5), rU = (Rg.get(F_RHO, nshift(n, 1, 1)) + r0) * R(0.5);
        const R rB = (r0 + rho_km1) * R(0.5), rF = (Rg.get(F_RHO, nshift(n, 2, 1)) + r0) * R(0.5);
        R e = R(0.);
#pragma unroll
        for (int q = 0; q < 3; q++) {
          const int a = AOFF + q;
          const R t = rR * gxb[(size_t)a * NXF + fxr] - rL * gxb[(size_t)a * NXF + fxl] +
                      rU * gyb[(size_t)a * NYF + fyu] - rD * gyb[(size_t)a * NYF + fyd] +
                      rF * (SMET ? gzr[a] : gzb[(size_t)a * NZF + fz]) - rB * Gzp[a];
          e = (q == 0) ? Rg.get(F_U + q, n) * t : e + Rg.get(F_U + q, n) * t;
        }
        return e;
      };
      const bool les_e = LES && VISC && ugj > 2 && ugj < c.my - 2 && nv < 0.5;
      double rhs[5];
      if (MIX) {
        // G = visc - conv' (FP32); the p_ref * h part of conv is p_ref * gcl (FP64)
        R d4[5];
#pragma unroll
        for (int q = 0; q < 5; q++) d4[q] = fdiff(q);
        if (les_e) d4[4] += les_energy();
        const double aj = aj_r;
        rhs[0] = (double)d4[0];
#pragma unroll
        for (int q = 1; q < 4; q++) rhs[q] = (double)d4[q] - c.p_ref * gcl_r[q - 1];
        rhs[4] = (double)d4[4];
        if (!PLAIN && c.twod == 1) rhs[1] = 0.;  // no x-momentum right-hand side (rhs.c:2135, 3168, 4215)
#pragma unroll
        for (int q = 0; q < 5; q++) rhs[q] = (nv < BLANK) ? rhs[q] * aj : 0.;
      } else {
        R conv[5], visc[5];
#pragma unroll
        for (int q = 0; q < 5; q++) conv[q] = (nv < BLANK) ? fdiff(q) : R(0.);
        visc[0] = R(0.);
#pragma unroll
        for (int q = 1; q < 5; q++) visc[q] = VISC ? fdiff(VOFF + q) : R(0.);
        if (!PLAIN && c.twod == 1) conv[1] = visc[1] = R(0.);  // rhs.c:2135-2140, 3168-3173, 4215-4220
        if (LES && nv < BLANK && c.ratio != 0.0) {  // channel forcing (rhs.c:4226-4235); exact no-op at ratio 0
          const double ajn = aj_r;
          conv[3] = conv[3] - c.ratio / ajn * Rg.get(F_RHO, n) / c.dt;
          conv[4] = conv[4] - c.ratio / ajn * Rg.get(F_RW, n) / c.dt;
        }
        if (les_e) visc[4] += les_energy();
        const double aj = aj_r;
#pragma unroll
        for (int q = 0; q < 5; q++) {
          rhs[q] = visc[q] - conv[q];                 // VecWAXPY(Rhs, -1, Conv, Visc)
          rhs[q] = (nv < BLANK) ? rhs[q] * aj : 0.;    // MultAj
        }
      }
      if (RHS_MODE) {
#pragma unroll
        for (int q = 0; q < 5; q++) F.rhs[q][g] = rhs[q];
      } else {
        double out[5];
#pragma unroll
        for (int q = 0; q < 5; q++) {
          const double qo = qo_r[q];
          const double qi = MIX ? qi_r[q] : (double)Rg.get(F_RHO + q, n);
          // solvers.c:257 (VecWAXPY) and 269 (VecAXPBYPCZ), FP64 in every form
          out[q] = (istage == 0) ? qo + adt * rhs[q] : beta * qo + adt * rhs[q] + alfa * qi;
          F.qout[q][g] = out[q];
        }
        const double p = (c.gamma - 1) * (out[4] - 0.5 * (out[1] * out[1] + out[2] * out[2] + out[3] * out[3]) / out[0]);
        unsigned st = 0;
        if (!isfinite(out[0] + out[1] + out[2] + out[3] + out[4])) st |= ST_NONFINITE;
        if (!(out[0] > 0.)) st |= ST_NEG_RHO;
        if (!(p > 0.)) st |= ST_NEG_P;
        if (st) atomicOr(F.status, st);
      }
#pragma unroll
      for (int q = 0; q < NG; q++) Gzp[q] = SMET ? gzr[q] : gzb[(size_t)q * NZF + fz];
    }
    base = base + 1 == NPL ? 0 : base + 1;
    if (SMET) cp_async_wait_all();  // the metric slot of plane k+1
    __syncthreads();
  }
}

// kchunk > 0: grid (tiles_x, tiles_y, k-chunks), one tile column and chunk
// per block.  kchunk == 0: balanced segments -- the tile columns' interior
// planes laid end to end (column after column) and cut into gridDim.x equal
// contiguous ranges, one per resident CTA; a CTA marches each column piece of
// its range with its own prologue.  Every node gets the same arithmetic in
// both shapes (a chunk start recomputes its first k-face from the same data).
template <typename R, bool MIX, bool LES, bool VISC, bool RHS_MODE, int FLUX = 0, bool NV0 = false>
static __global__ void __launch_bounds__(StageThreads<FLUX, MIX>::N, StageThreads<FLUX, MIX>::MIN_BLOCKS)
    stage_kernel(const DevCfg c, const DevFields F, int istage, double alfa, double beta, double adt, int kchunk) {
  extern __shared__ double smem_d[];
  constexpr int BY = StageGeo<FLUX>::BY;
  const int nk = c.mz - 2, tiles_x = (c.mx - 2 + SBX - 1) / SBX;
  long long s, e;  // range of (column, plane) units, column-major
  if (kchunk > 0) {
    const long long col = (long long)blockIdx.y * tiles_x + blockIdx.x;
    const int k0 = blockIdx.z * kchunk;
    s = col * nk + k0;
    e = col * nk + min(nk, k0 + kchunk);
  } else {
    const long long total = (long long)tiles_x * ((c.my - 2 + BY - 1) / BY) * nk;
    const long long per = (total + gridDim.x - 1) / gridDim.x;
    s = min(total, (long long)blockIdx.x * per);
    e = min(total, s + per);
  }
  while (s < e) {
    const int col = (int)(s / nk), k0 = (int)(s - (long long)col * nk);
    const int k1 = (int)min((long long)nk, k0 + (e - s));
    stage_tile<R, MIX, LES, VISC, RHS_MODE, FLUX, NV0>(c, F, col % tiles_x, col / tiles_x, 1 + k0, 1 + k1, istage, alfa,
                                                      beta, adt, smem_d);
    s += k1 - k0;
  }
}

// The time-step kernel without nvert (NV0) for FLUX bits fl: Roe, with LES
// the constant-sigma variants, and WENO5-JS; fl outside them runs the
// general blend.
using StageKern = void (*)(const DevCfg, const DevFields, int, double, double, double, int);
template <typename R, bool MIX, bool LES, bool VISC, int W>
static StageKern stage_nv0_kernel_w(int fl) {
  if constexpr (LES) {
    switch (fl & 7) {
      case 1: return stage_kernel<R, MIX, LES, VISC, false, W | 1, true>;
      case 2: return stage_kernel<R, MIX, LES, VISC, false, W | 2, true>;
      case 3: return stage_kernel<R, MIX, LES, VISC, false, W | 3, true>;
      case 4: return stage_kernel<R, MIX, LES, VISC, false, W | 4, true>;
      case 5: return stage_kernel<R, MIX, LES, VISC, false, W | 5, true>;
      default: return stage_kernel<R, MIX, LES, VISC, false, W, true>;
    }
  } else {
    return (fl & FLUX_ROE) ? stage_kernel<R, MIX, LES, VISC, false, W | 1, true> : stage_kernel<R, MIX, LES, VISC, false, W, true>;
  }
}
// (static, like the kernels: each object's selector returns its own kernels)
template <typename R, bool MIX, bool LES, bool VISC>
static StageKern stage_nv0_kernel(int fl) {
  switch (fl & (FLUX_W5 | FLUX_PLAIN)) {
    case FLUX_W5: return stage_nv0_kernel_w<R, MIX, LES, VISC, FLUX_W5>(fl);
    case FLUX_PLAIN: return stage_nv0_kernel_w<R, MIX, LES, VISC, FLUX_PLAIN>(fl);
    case FLUX_W5 | FLUX_PLAIN: return stage_nv0_kernel_w<R, MIX, LES, VISC, FLUX_W5 | FLUX_PLAIN>(fl);
    default: return stage_nv0_kernel_w<R, MIX, LES, VISC, 0>(fl);
  }
}
// The general (nvert-reading) kernel for the Roe and WENO5 bits of fl.
template <typename R, bool MIX, bool LES, bool VISC, bool RHSM>
static StageKern stage_gen_kernel(int fl) {
  switch (fl & (FLUX_ROE | FLUX_W5)) {
    case FLUX_ROE: return stage_kernel<R, MIX, LES, VISC, RHSM, FLUX_ROE>;
    case FLUX_W5: return stage_kernel<R, MIX, LES, VISC, RHSM, FLUX_W5>;
    case FLUX_ROE | FLUX_W5: return stage_kernel<R, MIX, LES, VISC, RHSM, FLUX_ROE | FLUX_W5>;
    default: return stage_kernel<R, MIX, LES, VISC, RHSM, 0>;
  }
}
// Threads and dynamic shared memory of a stage-kernel launch for FLUX bits fl.
template <bool MIX>
inline int stage_threads(int fl) {
  return (fl & FLUX_W5) ? StageThreads<FLUX_W5, MIX>::N : StageThreads<0, MIX>::N;
}
template <typename R, bool MIX>
size_t stage_smem_for(int fl, bool nv0) {
  const bool w5 = (fl & FLUX_W5) != 0;
  if (nv0) return w5 ? stage_smem<R, MIX, true, true>() : stage_smem<R, MIX, true, false>();
  return w5 ? stage_smem<R, MIX, false, true>() : stage_smem<R, MIX, false, false>();
}
// Opt every variant of one (LES, VISC, RHSM) into its dynamic shared memory.
template <typename R, bool MIX, bool LES, bool VISC, bool RHSM>
static cudaError_t stage_attrs() {
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaSuccess;
  for (int fl : {0, FLUX_ROE, FLUX_W5, FLUX_ROE | FLUX_W5})
    if (e == cudaSuccess) e = cudaFuncSetAttribute(stage_gen_kernel<R, MIX, LES, VISC, RHSM>(fl), attr, (int)stage_smem_for<R, MIX>(fl, false));
  if constexpr (!RHSM) {  // the no-IBM variants of the time step
    for (int w : {0, FLUX_W5, FLUX_PLAIN, FLUX_W5 | FLUX_PLAIN})
      for (int fl = 0; fl < (LES ? 6 : 2) && e == cudaSuccess; fl++)
        e = cudaFuncSetAttribute(stage_nv0_kernel<R, MIX, LES, VISC>(w | fl), attr, (int)stage_smem_for<R, MIX>(w | fl, true));
  }
  return e;
}

// ------------------------------------------------------- batched form ----
// Several blocks of uneven sizes advanced by ONE persistent launch: every CTA
// takes work items (block, tile column, k-chunk) from a device counter until
// the list is exhausted (a bounded loop, no waiting on other CTAs).  Items are
// listed largest-first by the host so the tail of the launch is short.  The
// blocks share the options, hence the FLUX bits and the tile geometry
// (StageGeo<FLUX>) the host cut the tile columns with.
struct BatchBlock {
  DevCfg c;
  DevFields F;
  int tiles_x, tiles_y, nchunks, kchunk;
  long long first_item;  // index of this block's first item in the global list
};

template <typename R, bool MIX, bool LES, bool VISC, bool NV0 = false, int FLUX = 0>
static __global__ void __launch_bounds__(StageThreads<FLUX, MIX>::N, StageThreads<FLUX, MIX>::MIN_BLOCKS)
    stage_batched_kernel(const BatchBlock *__restrict__ blocks, const int2 *__restrict__ items, int nitems,
                         unsigned *__restrict__ counter, int istage, double alfa, double beta, double adt) {
  extern __shared__ double smem_d[];
  __shared__ BatchBlock bb;
  __shared__ int item;
  for (;;) {
    if (threadIdx.x == 0) item = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int it = item;
    if (it >= nitems) break;
    const int2 ib = items[it];  // (block, local item index)
    if (threadIdx.x == 0) bb = blocks[ib.x];
    __syncthreads();
    const int txy = bb.tiles_x * bb.tiles_y;
    const int bzi = ib.y / txy, rem = ib.y - bzi * txy;
    const int byi = rem / bb.tiles_x, bxi = rem - byi * bb.tiles_x;
    const int kb = 1 + bzi * bb.kchunk;
    stage_tile<R, MIX, LES, VISC, false, FLUX, NV0>(bb.c, bb.F, bxi, byi, kb, min(bb.c.mz - 1, kb + bb.kchunk), istage,
                                                   alfa, beta, adt, smem_d);
    __syncthreads();  // bb and item are rewritten by the next iteration
  }
}

}  // namespace cb
