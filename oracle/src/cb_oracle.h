/*
 * CPU restatement of the reference's compressible RHS + SSP-RK stage update.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: tests/, the smoke entry
 * point and the CPU-baseline leg of bench.py may call it; the product never
 * links or calls it.
 *
 * Layout: every field is a separate plane (SoA) over the padded node box
 * (mx+4) x (my+4) x (mz+4): node (i,j,k) of the reference's DMDA, with
 * i in [-2, mx+1], lives at ((k+2)*(my+4) + (j+2))*(mx+4) + (i+2).  The two
 * ghost layers of a periodic direction hold the DMDA wrap-around copies
 * (index -1 -> mx-1, -2 -> mx-2, mx -> 0, mx+1 -> 1); those of a
 * non-periodic direction are unused.
 */
#ifndef CB_ORACLE_H
#define CB_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int mx, my, mz;          /* DMDA node counts including boundary nodes 0 and m-1 */
  int bctype[6];           /* bcs.dat codes, 7 = periodic */
  int les;                 /* -les: 0 off, 1 constant Smagorinsky, 3 dynamic node by node, 10 no model,
                              other values dynamic with local averaging */
  int inviscid;            /* -inv */
  int fluxorder;           /* -fluxorder: 1 first order, 2 MUSCL, 3 WENO3 */
  int eno_order;           /* -ENOorder */
  int central;             /* -central: 2 skew-symmetric, 3 Fp_1, other: 2-point */
  int isothermal;          /* -isothermal */
  double s_x, s_y, s_z;    /* -s_x/-s_y/-s_z hybrid weights */
  double ren, ma, pr, gamma, dt, st;
  double cs_const;         /* constant Smagorinsky coefficient (CS field value) */
  double ci;               /* Yoshizawa constant CI */
  double ratio;            /* channel forcing ratio (0 unless channel/wavy) */
  int calc_sigma;          /* -calc_sigma: pressure shock sensor for the hybrid weights */
  double s_x_min, s_y_min, s_z_min; /* -s_x_min/-s_y_min/-s_z_min: lower bounds of the sensor */
  double sigma_thrsh;      /* -sigma_thrsh: ks of the smoothness ratio (default 1e-5) */
  int flux;                /* upwind flux: 0 Rusanov (the reference's), 1 Roe with Harten's entropy fix */
  double max_cs;           /* -max_cs: upper clip of the dynamic Smagorinsky coefficient (default 0.05) */
  double twall;            /* -Twall: wall temperature of the characteristic isothermal wall (default 1) */
  int twod;                /* -twoD: 1 is the 2-D mode in i (no i-face fluxes, zero x-momentum
                              right-hand side, lUcat x = 0) and drops the x term of that wall (and x in the IB) */
  int i_homo_filter, j_homo_filter, k_homo_filter; /* -i/-j/-k_homo_filter: homogeneous averaging of the
                              dynamic model's LM and MM (les.c:916-1115) */
  int testfilter_ik;       /* -testfilter_ik: test-filter width 5^(1/3) instead of 2 filter widths (les.c:598) */
  int visT;                /* -visT: Sutherland's law for the molecular viscosity (rhs.c:1412-1414) */
  double tref;             /* -Tref: its reference temperature (default 273.15, rhs.c:1410) */
  int abc;                 /* -ABC: sensor weights 0 (then clamped) above plane k = ABC (rhs.c:3311, 3341-3368) */
  int weno_order;          /* 3: the reference's WENO3 (fluxorder 3); 5: WENO5-JS (Jiang & Shu 1996) where its
                              six-node stencil fits (no reference counterpart) */
  const double *coor_x;    /* node coordinates x and y (padded planes) for the k-lo inflow codes 52 and 47, */
  const double *coor_y;    /* which read them (rhs.c:854-874, 904-950); may be NULL otherwise */
  int ti0;                 /* user->ti of the first time step cbo_steps takes (the driver's first step is 1);
                              code 47 reads it */
} cbo_config;

/* WENO5-JS reconstruction at the face x_{i+1/2} from v_{i-2..i+2}, biased to
 * the left (the right-biased value at x_{i+1/2} is cbo_weno5(v_{i+3}, ...,
 * v_{i-1})).  Exposed for the known-answer tests of the reconstruction. */
double cbo_weno5(double a, double b, double c, double d, double e);

/* Fill the two ghost layers of each periodic direction of one padded plane
 * from the owned nodes by wrap-around (DMGlobalToLocal semantics). */
void cbo_fill_ghosts(const cbo_config *c, double *f);

/* FormMetrics: coordinates (3 padded planes) -> csi,eta,zet (3 planes each),
 * aj (1 plane); ghost layers of periodic directions filled. */
void cbo_metrics(const cbo_config *c, const double *const coor[3], double *const csi[3],
                 double *const eta[3], double *const zet[3], double *aj);

/* EqOfState on every node of the padded box. */
void cbo_eos(const cbo_config *c, const double *const q[5], double *p);

/* Hybrid weights field (3 planes) as formConvectionLES sets it at istage 0
 * when the sensor is off. */
void cbo_sigma(const cbo_config *c, double *const sig[3]);

/* Hybrid weights with the pressure shock sensor (-calc_sigma 1), as
 * formConvectionLES sets them at istage 0 from the ghosted stage state q. */
void cbo_sigma_sensor(const cbo_config *c, const double *const q[5], double *const sig[3]);
/* The same from a ghosted pressure p (the lP formConvectionLES reads: after
 * an immersed step, the pressure carried from the interpolation). */
void cbo_sigma_sensor_p(const cbo_config *c, const double *p, double *const sig[3]);

/* formRHS: q = ghosted stage state, nut/sig may be NULL when les == 0.
 * rhs: 5 padded planes; interior nodes written, every other node zeroed. */
int cbo_rhs(const cbo_config *c, const double *const q[5], const double *const csi[3],
            const double *const eta[3], const double *const zet[3], const double *aj,
            const double *nvert, const double *nut, const double *const sig[3],
            double *const rhs[5]);

/* Compute_eddy_viscosity_LES: u from the ghosted state qu (NULL: zero
 * velocity, as before the first CalcUCat), nut written on interior nodes,
 * boundary nodes untouched, then ghost layers refreshed. */
void cbo_eddy_viscosity(const cbo_config *c, const double *const qu[5], const double *const csi[3],
                        const double *const eta[3], const double *const zet[3], const double *aj,
                        const double *nvert, double *nut);

/* One SSP-RK stage update on every node: qout = combination of qold, qin, rhs. */
void cbo_rk_combine(const cbo_config *c, int istage, const double *const qold[5],
                    const double *const qin[5], const double *const rhs[5], double *const qout[5]);

/* FormBCS periodic part: boundary nodes of qout from the stale ghosted stage
 * input qin, then DMGlobalToLocal of qout. */
int cbo_bc_periodic(const cbo_config *c, const double *const qin[5], double *const qout[5]);

/* FormBCS: boundary nodes of q (the RK-combined stage output) from the
 * boundary codes, the periodic copies from the stale ghosted stage input lq,
 * then the ghost wrap; alfa: the stage's RK coefficient.  Returns 5 for the
 * codes that are not restated. */
int cbo_formbcs(const cbo_config *c, double alfa, const double *const lq[5], const double *const qold[5],
                const double *const eta[3], const double *const zet[3], const double *aj, const double *nvert,
                double *const q[5]);

/* Full time steps (Flow_Solver + main loop): q (ghosted, in/out), qold,
 * quc (ghosted state of the last CalcUCat; in/out), have_uc (in/out flag),
 * nut (in/out).  Scratch buffers are allocated inside. */
int cbo_steps(const cbo_config *c, int nsteps, double *const q[5], double *const qold[5],
              double *const quc[5], int *have_uc, double *nut, const double *const csi[3],
              const double *const eta[3], const double *const zet[3], const double *aj,
              const double *nvert);

/* One entry of the immersed-boundary interpolation list (IBMInfo,
 * variables.h:50-89): the interface node, the surface element of its
 * interception point (-1: none), three donor nodes with weights cr, the
 * element's vertex weights cs, the distances node -> surface (d_s) and
 * surface -> donor point (d_i), and the interception point pmin. */
typedef struct {
  int ni, nj, nk, cell;
  int i1, j1, k1, i2, j2, k2, i3, j3, k3;
  int pad;
  double cr1, cr2, cr3, cs1, cs2, cs3, d_s, d_i, pmin[3];
} cbo_ibm_info;

/* The surface arrays of one body the interpolation reads (IBMNodes,
 * variables.h:91-118): triangles, their normals, the vertex velocities of
 * this and the previous step (x, y, z per vertex). */
typedef struct {
  int n_v, n_elmt;
  const int *nv1, *nv2, *nv3;
  const double *nf_x, *nf_y, *nf_z;
  const double *u, *uold;
} cbo_ibm_surface;

/* ibm_interpolation_advanced (ibm_iso.c:2572-2880): five Jacobi sweeps over
 * the list; q (ghosted, in/out) serves as both Q and lQ, p (ghosted, in/out)
 * as P and lP, coor the node coordinates (3 padded planes), qold the step's
 * start state whose density the characteristic wall of -isothermal 2 reads
 * (NULL: q as given).  wallfunction 0 (noslip, freeslip with -inv), 2 (the
 * hydset log law; ustar, if not NULL, receives u_tau of every entry from the
 * last sweep) or 3 (freeslip).  Returns 5 for wall function 1, which is not
 * restated. */
int cbo_ibm_interpolate(const cbo_config *c, const cbo_ibm_surface *s, int n, const cbo_ibm_info *list,
                        const double *const coor[3], double *const q[5], double *p, const double *const qold[5],
                        int add_dundt, int twoD, int wallfunction, double *ustar);

/* formRHS / FormBCS reading the local pressure lp (padded) the reference
 * carries in lP instead of the EqOfState of the stage input; cbo_formbcs_lp
 * also copies P (p, in/out; may be NULL) across periodic boundaries from lp
 * and wraps its ghosts, as FormBCS does (rhs.c:1107-1227, 1305-1308). */
int cbo_rhs_lp(const cbo_config *c, const double *const q[5], const double *lp, const double *const csi[3],
               const double *const eta[3], const double *const zet[3], const double *aj,
               const double *nvert, const double *nut, const double *const sig[3],
               double *const rhs[5]);
int cbo_formbcs_lp(const cbo_config *c, double alfa, const double *const lq[5], const double *lp,
                   const double *const qold[5], const double *const eta[3], const double *const zet[3],
                   const double *aj, const double *nvert, double *const q[5], double *p);

/* Time steps with immersed bodies (RungeKutta with -imm): the stages, the
 * interpolation of each of the nbodies bodies (surf[b], lists[b] with
 * nlist[b] entries), then FormBCS(user, 0).  lp (padded, in/out) is the
 * pressure the reference keeps in P / lP; *lp_valid (in/out) says whether
 * the first stage reads it (set after an immersed step) or the EqOfState of
 * its input.  Returns 5 with the shock sensor (not restated here). */
int cbo_steps_ibm(const cbo_config *c, int nsteps, double *const q[5], double *const qold[5],
                  double *const quc[5], int *have_uc, double *nut, const double *const csi[3],
                  const double *const eta[3], const double *const zet[3], const double *aj,
                  const double *nvert, int nbodies, const cbo_ibm_surface *surf, const int *nlist,
                  const cbo_ibm_info *const *lists, const double *const coor[3], double *lp, int *lp_valid,
                  int twoD, int wallfunction);

/* The dynamic model runs: -les >= 2 except 10 (les.c:138-146 single out 1
 * and 10; solvers.c:28 skips the model with 10). */
int cbo_les_dynamic(const cbo_config *c);

/* Compute_Smagorinsky_Constant_1 with a dynamic -les (les.c:151-1472, the
 * 3-D box test filter; local 27-node averaging, or LM / MM node by node with
 * -les 3 or a homogeneous filter, which also adds the plane / line / box
 * averages of -i/-j/-k_homo_filter): Cs per node into cs (global CS, in/out:
 * boundary nodes keep their value through the clipping) from the ghosted
 * current state q, the state quc of the last CalcUCat (NULL: zero velocity)
 * and the local pressure lp.  Returns 5 unless cbo_les_dynamic. */
int cbo_dynamic_smagorinsky(const cbo_config *c, const double *const q[5], const double *const quc[5],
                            const double *lp, const double *const csi[3], const double *const eta[3],
                            const double *const zet[3], const double *aj, const double *nvert, double *cs);
/* Compute_eddy_viscosity_LES after the dynamic model: Cs per node, and the
 * velocity the model left in lUcat (q at interior nodes with nvert <= 1.1,
 * quc elsewhere). */
void cbo_eddy_viscosity_dyn(const cbo_config *c, const double *const q[5], const double *const quc[5],
                            const double *const csi[3], const double *const eta[3], const double *const zet[3],
                            const double *aj, const double *nvert, const double *cs, double *nut);

/* Number of RK stages the reference runs for this config (= fluxorder). */
int cbo_nstages(const cbo_config *c);

#ifdef __cplusplus
}
#endif
#endif
