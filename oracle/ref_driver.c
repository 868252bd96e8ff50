/*
 * Driver that runs the reference's own hot-path source (rhs.c, les.c,
 * metrics.c, solvers.c, and the immersed boundary's ibm_iso.c, compgeom.c,
 * variables.c, wallfunction.c, compiled UNMODIFIED against the serial PETSc shim)
 * behind a small C-ABI, so tests can pin the oracle restatement and the CUDA
 * path against the reference's actual arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  Built into oracle/_ref/libchimera_ref.so by
 * oracle/Makefile; never linked by the product.
 *
 * What it mirrors from the reference (no code copied, only the call order):
 *   main.c:14-75        global option variables and their defaults
 *   main.c:716-801      option parsing into those globals
 *   init.c:105-220      DMDA creation (stencil width 2, periodic per bctype)
 *   init.c:956-1090     vector allocation
 *   init.c:45-103       FormInitialize defaults (-ren/-Ma/-Pr/-gamma/-dt)
 *   rhs.c:420-433       tail of SetInitialCondition (lQ scatter, Qold, EOS)
 *   main.c:887-974      time loop: ti from tistart+1, Flow_Solver, Q -> Qold
 * Functions called from the reference: FormMetrics (metrics.c:3),
 * EqOfState (rhs.c:4820), CalcUCat (rhs.c:1322), formRHS (rhs.c:4703),
 * FormBCS (rhs.c:477), Compute_Smagorinsky_Constant_1 (les.c:135),
 * Compute_eddy_viscosity_LES (les.c:1477), RungeKutta (solvers.c:223),
 * Flow_Solver (solvers.c:13), ibm_search_advanced (ibm_iso.c:87),
 * ibm_interpolation_advanced (ibm_iso.c:2572).
 */
#include "variables.h"

/* ---- globals the reference expects from main.c (defaults main.c:14-75) ----
 * With CHIMERA_REF_WITH_MAIN the reference's main.c itself is linked (its
 * checkpoint writer/reader and RestartApplication, main.c:215-304, 620-693)
 * and defines these; the driver then keeps only those main.c lacks. */
#ifndef CHIMERA_REF_WITH_MAIN
PetscInt tistart = 0;
PetscBool rstart_flg = PETSC_FALSE;
PetscInt immersed = 0;
PetscInt wavy = 0, isothermal = 0;
PetscInt calc_sigma = 0;
PetscInt invicid = 0;
PetscInt movefsi = 0, rotatefsi = 0, sediment = 0;
PetscReal CMx_c = 0., CMy_c = 0., CMz_c = 0.;
PetscInt TwoD = 0;
PetscInt STRONG_COUPLING = 0;
PetscInt fish = 0;
PetscInt NumberOfBodies = 1;
PetscInt moveframe = 0, rotateframe = 0;
PetscInt central = 2;
PetscInt les = 0, rans = 0;
PetscInt wallfunction = 0;
PetscInt averaging = 0;
PetscInt mixed = 0;
PetscInt clark = 0;
PetscInt dynamic_freq = 1;
PetscInt i_periodic = 0, j_periodic = 0, k_periodic = 0;
PetscInt ii_periodic = 0, jj_periodic = 0, kk_periodic = 0;
PetscInt testfilter_ik = 0, testfilter_1d = 0;
PetscInt i_homo_filter = 0, j_homo_filter = 0, k_homo_filter = 0;
PetscInt channel = 0;
PetscInt block_number = 1;
PetscReal max_cs = 0.5;
PetscInt thin = 0;  /* main.c:45, read by ibm_search_advanced */
#else
extern PetscInt tistart;
extern PetscBool rstart_flg;
extern PetscInt immersed, wavy, isothermal, calc_sigma, invicid, movefsi, rotatefsi, sediment;
extern PetscReal CMx_c, CMy_c, CMz_c;
extern PetscInt TwoD, STRONG_COUPLING, fish, NumberOfBodies, moveframe, rotateframe, central, les, rans;
extern PetscInt wallfunction, averaging, mixed, clark, dynamic_freq, i_periodic, j_periodic, k_periodic;
extern PetscInt testfilter_ik, testfilter_1d, i_homo_filter, j_homo_filter, k_homo_filter, channel, thin;
extern PetscReal max_cs;
PetscInt ii_periodic = 0, jj_periodic = 0, kk_periodic = 0;
PetscInt block_number = 1;
#endif

/* ---- reference entry points (prototypes live only under __cplusplus) ---- */
PetscErrorCode FormMetrics(UserCtx *user);
PetscErrorCode EqOfState(UserCtx *user);
PetscErrorCode CalcUCat(UserCtx *user);
PetscErrorCode formRHS(UserCtx *user, Vec Rhs, PetscInt istage);
PetscErrorCode FormBCS(UserCtx *user, PetscReal alfa);
void Compute_Smagorinsky_Constant_1(UserCtx *user);
void Compute_eddy_viscosity_LES(UserCtx *user);
PetscErrorCode RungeKutta(UserCtx *user, IBMNodes *ibm, FSInfo *fsi);
PetscErrorCode Flow_Solver(UserMG *usermg, IBMNodes *ibm, FSInfo *fsi);
PetscErrorCode ibm_search_advanced(UserCtx *user, IBMNodes *ibm, PetscInt ibi);
PetscErrorCode ibm_interpolation_advanced(UserCtx *user, IBMNodes *ibm, PetscInt ibi, PetscInt Add_dUndt);
void InitIBMList(IBMList *ilist);
void AddIBMNode(IBMList *ilist, IBMInfo ibm_intp);
void DestroyIBMList(IBMList *ilist);

/* ---- stubs for subsystems outside the hot path (IBM, FSI, output) ---- */
#ifndef CHIMERA_REF_WITH_MAIN
PetscErrorCode Q_P_Binary_Output(UserCtx *u) { (void)u; return 0; }
#endif
PetscErrorCode Calc_forces_SI2() { return 0; }
PetscErrorCode Calc_FSI_pos_intg() { return 0; }
PetscErrorCode fish_swim() { return 0; }
PetscErrorCode Elmt_Move_FSI_TRANSpROT_quarternion() { return 0; }
PetscErrorCode calc_ibm_normal() { return 0; }
PetscErrorCode Elmt_Move_FSI_TRANS() { return 0; }
PetscErrorCode Set_ibm_velocity_to_fsi() { return 0; }
PetscErrorCode ibm_surface_VTKOut() { return 0; }
PetscErrorCode FSI_position_Output() { return 0; }
PetscErrorCode FSI_DATA_Output() { return 0; }

/* ---- driver state ---- */
static UserCtx *U = NULL;
static UserMG MG;
static MGCtx MGC;
static PetscInt g_ti = 0;
static IBMNodes *IBM = NULL;  /* one immersed body (ibi 0) */

static void read_globals_from_options(void) {
  /* main.c:716-801 (subset that the hot path reads) */
  PetscOptionsGetInt(NULL, NULL, "-imm", &immersed, NULL);
  PetscOptionsGetInt(NULL, NULL, "-wavy", &wavy, NULL);
  PetscOptionsGetInt(NULL, NULL, "-isothermal", &isothermal, NULL);
  PetscOptionsGetInt(NULL, NULL, "-inv", &invicid, NULL);
  PetscOptionsGetInt(NULL, NULL, "-TwoD", &TwoD, NULL);
  PetscOptionsGetInt(NULL, NULL, "-les", &les, NULL);
  PetscOptionsGetInt(NULL, NULL, "-rans", &rans, NULL);
  PetscOptionsGetInt(NULL, NULL, "-central", &central, NULL);
  PetscOptionsGetInt(NULL, NULL, "-channel", &channel, NULL);
  PetscOptionsGetInt(NULL, NULL, "-calc_sigma", &calc_sigma, NULL);
  PetscOptionsGetInt(NULL, NULL, "-wallfunction", &wallfunction, NULL);
  PetscOptionsGetInt(NULL, NULL, "-thin", &thin, NULL);
  PetscOptionsGetInt(NULL, NULL, "-clark", &clark, NULL);
  PetscOptionsGetInt(NULL, NULL, "-testfilter_ik", &testfilter_ik, NULL);
  PetscOptionsGetInt(NULL, NULL, "-testfilter_1d", &testfilter_1d, NULL);
  PetscOptionsGetInt(NULL, NULL, "-i_homo_filter", &i_homo_filter, NULL);
  PetscOptionsGetInt(NULL, NULL, "-j_homo_filter", &j_homo_filter, NULL);
  PetscOptionsGetInt(NULL, NULL, "-k_homo_filter", &k_homo_filter, NULL);
}

static void reset_globals(void) {
  tistart = 0; rstart_flg = PETSC_FALSE; immersed = 0; wavy = 0; isothermal = 0;
  calc_sigma = 0; invicid = 0; TwoD = 0; central = 2; les = 0; rans = 0; channel = 0;
  wallfunction = 0; thin = 0; clark = 0; testfilter_ik = 0; testfilter_1d = 0;
  i_homo_filter = 0; j_homo_filter = 0; k_homo_filter = 0;
}

static void ibm_free(void) {
  if (U && U->ibmlist) {
    DestroyIBMList(&U->ibmlist[0]);
    free(U->ibmlist);
    U->ibmlist = NULL;
  }
  if (!IBM) return;
  void *arrs[] = {IBM->x_bp, IBM->y_bp, IBM->z_bp, IBM->nv1, IBM->nv2, IBM->nv3, IBM->nf_x, IBM->nf_y,
                  IBM->nf_z, IBM->u, IBM->uold, IBM->urm1};
  for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); i++) free(arrs[i]);
  free(IBM);
  IBM = NULL;
}

static void destroy_user(void) {
  ibm_free();
  if (!U) return;
  Vec *vs[] = {&U->Q, &U->Qold, &U->Rhs, &U->lQ, &U->lQold, &U->Ucat, &U->Nvert, &U->P, &U->Nvert_o,
               &U->lCsi, &U->lEta, &U->lZet, &U->lUcat, &U->lAj, &U->lNvert, &U->lP, &U->lNvert_o,
               &U->lBeta, &U->Sigma, &U->lSigma, &U->lNu_t, &U->Nu_t, &U->lCS, &U->CS, &U->lBBeta, &U->lUstar};
  for (size_t i = 0; i < sizeof(vs) / sizeof(vs[0]); i++) VecDestroy(vs[i]);
  DMDestroy(&U->cda);
  DMDestroy(&U->da);
  free(U);
  U = NULL;
}

/* options: whitespace separated "-name value" pairs, as on the reference's
 * command line.  coords: AoS (x,y,z) per node, natural k-j-i order. */
int ref_setup(int mx, int my, int mz, const int *bctype, const double *coords, const char *options) {
  destroy_user();
  reset_globals();
  shim_options_clear();
  if (options) {
    char buf[4096];
    snprintf(buf, sizeof(buf), "%s", options);
    char *save = NULL;
    char *tok = strtok_r(buf, " \t\n", &save);
    while (tok) {
      char *name = tok;
      char *val = strtok_r(NULL, " \t\n", &save);
      if (shim_options_set(name, val ? val : "")) return 2;
      tok = val ? strtok_r(NULL, " \t\n", &save) : NULL;
    }
  }
  read_globals_from_options();

  U = (UserCtx *)calloc(1, sizeof(UserCtx));
  for (int b = 0; b < 6; b++) U->bctype[b] = bctype[b];
  U->IM = mx; U->JM = my; U->KM = mz;
  U->block_number = 1;
  U->thislevel = 0;
  U->mglevels = 1;
  U->tiout = 1 << 30;

  /* init.c:148-199: periodic flags from bctype */
  DMBoundaryType xp = DM_BOUNDARY_NONE, yp = DM_BOUNDARY_NONE, zp = DM_BOUNDARY_NONE;
  int b0 = U->bctype[0] == 7, b2 = U->bctype[2] == 7, b4 = U->bctype[4] == 7;
  if (b0 && b2 && b4) { xp = yp = zp = DM_BOUNDARY_PERIODIC; }
  else if (b0 && b2) { xp = yp = DM_BOUNDARY_PERIODIC; }
  else if (b2 && b4) { yp = zp = DM_BOUNDARY_PERIODIC; }
  else if (b0 && b4) { xp = zp = DM_BOUNDARY_PERIODIC; }
  else if (b0) { xp = DM_BOUNDARY_PERIODIC; }
  else if (b2) { yp = DM_BOUNDARY_PERIODIC; }
  else if (b4) { zp = DM_BOUNDARY_PERIODIC; }
  DMDACreate3d(PETSC_COMM_WORLD, xp, yp, zp, DMDA_STENCIL_BOX, mx, my, mz, 1, 1, 1, 1, 2, NULL, NULL, NULL, &U->da);
  DMDACreate3d(PETSC_COMM_WORLD, xp, yp, zp, DMDA_STENCIL_BOX, mx, my, mz, 1, 1, 1, 5, 2, NULL, NULL, NULL, &U->cda);
  DMDASetUniformCoordinates(U->da, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0);
  DMGetCoordinateDM(U->da, &U->fda);
  DMDAGetLocalInfo(U->da, &U->info);
  if (coords) {
    Vec c;
    DMGetCoordinates(U->da, &c);
    memcpy(c->a, coords, sizeof(double) * 3 * (size_t)mx * my * mz);
  }

  /* init.c:956-1090 allocation */
  DMCreateGlobalVector(U->cda, &U->Q);
  VecDuplicate(U->Q, &U->Qold);
  VecDuplicate(U->Q, &U->Rhs);
  DMCreateLocalVector(U->cda, &U->lQ);
  VecDuplicate(U->lQ, &U->lQold);
  DMCreateGlobalVector(U->fda, &U->Csi);
  VecDuplicate(U->Csi, &U->Eta);
  VecDuplicate(U->Csi, &U->Zet);
  VecDuplicate(U->Csi, &U->Ucat);
  DMCreateGlobalVector(U->da, &U->Aj);
  VecDuplicate(U->Aj, &U->Nvert);
  VecDuplicate(U->Aj, &U->P);
  VecDuplicate(U->Aj, &U->Nvert_o);
  DMCreateLocalVector(U->fda, &U->lCsi);
  VecDuplicate(U->lCsi, &U->lEta);
  VecDuplicate(U->lCsi, &U->lZet);
  VecDuplicate(U->lCsi, &U->lUcat);
  DMCreateLocalVector(U->da, &U->lAj);
  VecDuplicate(U->lAj, &U->lNvert);
  if (les) {
    VecDuplicate(U->lCsi, &U->lBeta);
    VecDuplicate(U->Csi, &U->Sigma);
    VecDuplicate(U->lCsi, &U->lSigma);
    VecDuplicate(U->lAj, &U->lNu_t);
    VecDuplicate(U->Aj, &U->Nu_t);
    VecDuplicate(U->lAj, &U->lCS);
    VecDuplicate(U->Aj, &U->CS);
    VecDuplicate(U->lAj, &U->lBBeta);
    VecSet(U->lNu_t, 0);
  }
  VecDuplicate(U->lAj, &U->lP);
  VecDuplicate(U->lAj, &U->lNvert_o);
  if (wallfunction) VecDuplicate(U->lAj, &U->lUstar); /* ibm_iso.c:2635 */

  /* init.c:45-103 FormInitialize */
  VecSet(U->Nvert, 0.); VecSet(U->lNvert, 0.);
  VecSet(U->P, 0.); VecSet(U->lP, 0.);
  VecSet(U->Nvert_o, 0.); VecSet(U->lNvert_o, 0.);
  U->FluxIntpSum = 0.; U->FluxInSum = 0.; U->FluxIntfcSum = 0.; U->FluxOutSum = 0.; U->ratio = 0.;
  U->ren = 3000.; U->Ma = 2.81; U->gamma = 1.4; U->Pr = 0.72; U->dt = 0.01; U->cfl = 0.2; U->vnn = 0.2;
  PetscOptionsGetReal(NULL, NULL, "-ren", &U->ren, NULL);
  PetscOptionsGetReal(NULL, NULL, "-Ma", &U->Ma, NULL);
  PetscOptionsGetReal(NULL, NULL, "-Pr", &U->Pr, NULL);
  PetscOptionsGetReal(NULL, NULL, "-gamma", &U->gamma, NULL);
  PetscOptionsGetReal(NULL, NULL, "-dt", &U->dt, NULL);
  PetscOptionsGetReal(NULL, NULL, "-cfl", &U->cfl, NULL);
  PetscOptionsGetReal(NULL, NULL, "-vnn", &U->vnn, NULL);
  U->st = 1.;

  FormMetrics(U);

  MGC.user = U;
  MGC.thislevel = 0;
  MG.mglevels = 1;
  MG.thislevel = 0;
  MG.mgctx = &MGC;
  /* main.c:887-892: tistart is incremented once before the time loop */
  tistart = 1;
  g_ti = tistart;
  return 0;
}

/* nvert: one value per node (natural order) */
int ref_set_nvert(const double *nvert) {
  if (!U) return 1;
  memcpy(U->Nvert->a, nvert, sizeof(double) * (size_t)U->Nvert->n);
  DMGlobalToLocalBegin(U->da, U->Nvert, INSERT_VALUES, U->lNvert);
  DMGlobalToLocalEnd(U->da, U->Nvert, INSERT_VALUES, U->lNvert);
  return 0;
}

/* Q: AoS 5 doubles per node.  Mirrors the tail of SetInitialCondition
 * (rhs.c:420-433): lQ <- Q, Qold <- Q, lQold <- lQ, EqOfState. */
int ref_set_state(const double *Q) {
  if (!U) return 1;
  memcpy(U->Q->a, Q, sizeof(double) * (size_t)U->Q->n);
  DMGlobalToLocalBegin(U->cda, U->Q, INSERT_VALUES, U->lQ);
  DMGlobalToLocalEnd(U->cda, U->Q, INSERT_VALUES, U->lQ);
  VecCopy(U->Q, U->Qold);
  VecCopy(U->lQ, U->lQold);
  EqOfState(U);
  return 0;
}

/* Overwrite the ghosted local state lQ (e.g. to reproduce a stale halo). */
int ref_set_local_state(const double *lQ) {
  if (!U) return 1;
  memcpy(U->lQ->a, lQ, sizeof(double) * (size_t)U->lQ->n);
  return 0;
}

int ref_set_nut(const double *nut) {
  if (!U || !U->Nu_t) return 1;
  memcpy(U->Nu_t->a, nut, sizeof(double) * (size_t)U->Nu_t->n);
  DMGlobalToLocalBegin(U->da, U->Nu_t, INSERT_VALUES, U->lNu_t);
  DMGlobalToLocalEnd(U->da, U->Nu_t, INSERT_VALUES, U->lNu_t);
  return 0;
}

int ref_calc_ucat(void) { if (!U) return 1; return CalcUCat(U); }

int ref_eddy_viscosity(void) {
  if (!U || !les) return 1;
  U->ti = g_ti;
  Compute_Smagorinsky_Constant_1(U);
  Compute_eddy_viscosity_LES(U);
  return 0;
}

/* formRHS(user, Rhs, istage); out: AoS 5 per node (global Rhs). */
int ref_rhs(int istage, double *rhs_out) {
  if (!U) return 1;
  U->ti = g_ti;
  int e = formRHS(U, U->Rhs, istage);
  if (rhs_out) memcpy(rhs_out, U->Rhs->a, sizeof(double) * (size_t)U->Rhs->n);
  return e;
}

/* nsteps physical time steps exactly as main.c:900-974 drives them. */
int ref_steps(int nsteps) {
  if (!U) return 1;
  for (int n = 0; n < nsteps; n++) {
    U->ti = g_ti;
    Flow_Solver(&MG, immersed ? IBM : NULL, NULL);
    VecCopy(U->Q, U->Qold);
    DMGlobalToLocalBegin(U->cda, U->Qold, INSERT_VALUES, U->lQold);
    DMGlobalToLocalEnd(U->cda, U->Qold, INSERT_VALUES, U->lQold);
    g_ti++;
  }
  return 0;
}

int ref_local_dims(int *gx, int *gy, int *gz) {
  if (!U) return 1;
  DMDALocalInfo in;
  DMDAGetLocalInfo(U->da, &in);
  *gx = in.gxm; *gy = in.gym; *gz = in.gzm;
  return 0;
}

static int copy_out(Vec v, double *out) {
  if (!v) return 1;
  memcpy(out, v->a, sizeof(double) * (size_t)v->n);
  return 0;
}

int ref_get_Q(double *out) { return U ? copy_out(U->Q, out) : 1; }
int ref_get_P(double *out) { return U ? copy_out(U->P, out) : 1; }
int ref_get_lQ(double *out) { return U ? copy_out(U->lQ, out) : 1; }
int ref_get_lP(double *out) { return U ? copy_out(U->lP, out) : 1; }
int ref_get_nut(double *out) { return U ? copy_out(U->Nu_t, out) : 1; }
int ref_get_cs(double *out) { return U && U->CS ? copy_out(U->CS, out) : 1; }
int ref_get_lnut(double *out) { return U ? copy_out(U->lNu_t, out) : 1; }
int ref_get_lsigma(double *out) { return U ? copy_out(U->lSigma, out) : 1; }
int ref_get_lucat(double *out) { return U ? copy_out(U->lUcat, out) : 1; }
int ref_get_metrics(double *lcsi, double *leta, double *lzet, double *laj) {
  if (!U) return 1;
  copy_out(U->lCsi, lcsi);
  copy_out(U->lEta, leta);
  copy_out(U->lZet, lzet);
  copy_out(U->lAj, laj);
  return 0;
}
void ref_destroy(void) { destroy_user(); }

/* ---- immersed boundary: one body, ibi 0 (main.c:813-858 sets up the same
 * objects: a calloc'ed IBMNodes, user->ibmlist with InitIBMList, the surface
 * as ibm_read_ucd leaves it, zero surface velocity) ---- */
int ref_ibm_setup(int n_v, int n_elmt, const double *x, const double *y, const double *z, const int *nv1,
                  const int *nv2, const int *nv3, const double *nf_x, const double *nf_y, const double *nf_z) {
  if (!U) return 1;
  ibm_free();
  IBM = (IBMNodes *)calloc(1, sizeof(IBMNodes));
  IBM->n_v = n_v;
  IBM->n_elmt = n_elmt;
  IBM->x_bp = malloc(sizeof(double) * n_v); memcpy(IBM->x_bp, x, sizeof(double) * n_v);
  IBM->y_bp = malloc(sizeof(double) * n_v); memcpy(IBM->y_bp, y, sizeof(double) * n_v);
  IBM->z_bp = malloc(sizeof(double) * n_v); memcpy(IBM->z_bp, z, sizeof(double) * n_v);
  IBM->nv1 = malloc(sizeof(PetscInt) * n_elmt); memcpy(IBM->nv1, nv1, sizeof(PetscInt) * n_elmt);
  IBM->nv2 = malloc(sizeof(PetscInt) * n_elmt); memcpy(IBM->nv2, nv2, sizeof(PetscInt) * n_elmt);
  IBM->nv3 = malloc(sizeof(PetscInt) * n_elmt); memcpy(IBM->nv3, nv3, sizeof(PetscInt) * n_elmt);
  IBM->nf_x = malloc(sizeof(double) * n_elmt); memcpy(IBM->nf_x, nf_x, sizeof(double) * n_elmt);
  IBM->nf_y = malloc(sizeof(double) * n_elmt); memcpy(IBM->nf_y, nf_y, sizeof(double) * n_elmt);
  IBM->nf_z = malloc(sizeof(double) * n_elmt); memcpy(IBM->nf_z, nf_z, sizeof(double) * n_elmt);
  IBM->u = calloc(n_v, sizeof(Cmpnts));
  IBM->uold = calloc(n_v, sizeof(Cmpnts));
  IBM->urm1 = calloc(n_v, sizeof(Cmpnts));
  U->ibmlist = (IBMList *)malloc(sizeof(IBMList));
  InitIBMList(&U->ibmlist[0]);
  return 0;
}

/* Surface velocity of the current and the previous step (n_v x,y,z each). */
int ref_ibm_set_velocity(const double *u, const double *uold) {
  if (!IBM) return 1;
  memcpy(IBM->u, u, sizeof(Cmpnts) * IBM->n_v);
  memcpy(IBM->uold, uold, sizeof(Cmpnts) * IBM->n_v);
  return 0;
}

/* ibm_search_advanced (ibm_iso.c:87): nvert and the interpolation list. */
int ref_ibm_search(void) {
  if (!U || !IBM) return 1;
  DestroyIBMList(&U->ibmlist[0]);
  InitIBMList(&U->ibmlist[0]);
  return ibm_search_advanced(U, IBM, 0);
}

int ref_get_nvert(double *out) { return U ? copy_out(U->Nvert, out) : 1; }

int ref_ibm_list_count(void) {
  if (!U || !U->ibmlist) return -1;
  int n = 0;
  for (IBMListNode *c = U->ibmlist[0].head; c; c = c->next) n++;
  return n;
}

/* The list in traversal order; per entry 13 ints (ni nj nk cell i1 j1 k1 i2 j2
 * k2 i3 j3 k3) and 11 doubles (cr1 cr2 cr3 cs1 cs2 cs3 d_s d_i pmin.x pmin.y
 * pmin.z). */
int ref_ibm_list_get(int *iv, double *rv) {
  if (!U || !U->ibmlist) return 1;
  int n = 0;
  for (IBMListNode *c = U->ibmlist[0].head; c; c = c->next, n++) {
    const IBMInfo *b = &c->ibm_intp;
    int *a = iv + 13 * n;
    double *r = rv + 11 * n;
    a[0] = b->ni; a[1] = b->nj; a[2] = b->nk; a[3] = b->cell;
    a[4] = b->i1; a[5] = b->j1; a[6] = b->k1; a[7] = b->i2; a[8] = b->j2; a[9] = b->k2;
    a[10] = b->i3; a[11] = b->j3; a[12] = b->k3;
    r[0] = b->cr1; r[1] = b->cr2; r[2] = b->cr3; r[3] = b->cs1; r[4] = b->cs2; r[5] = b->cs3;
    r[6] = b->d_s; r[7] = b->d_i; r[8] = b->pmin.x; r[9] = b->pmin.y; r[10] = b->pmin.z;
  }
  return 0;
}

/* Replace the list (same per-entry layout as ref_ibm_list_get, traversal
 * order kept: AddIBMNode prepends, so entries are added last to first). */
int ref_ibm_list_set(int n, const int *iv, const double *rv) {
  if (!U || !U->ibmlist) return 1;
  DestroyIBMList(&U->ibmlist[0]);
  InitIBMList(&U->ibmlist[0]);
  for (int e = n - 1; e >= 0; e--) {
    IBMInfo b;
    memset(&b, 0, sizeof(b));
    const int *a = iv + 13 * e;
    const double *r = rv + 11 * e;
    b.ni = a[0]; b.nj = a[1]; b.nk = a[2]; b.cell = a[3];
    b.i1 = a[4]; b.j1 = a[5]; b.k1 = a[6]; b.i2 = a[7]; b.j2 = a[8]; b.k2 = a[9];
    b.i3 = a[10]; b.j3 = a[11]; b.k3 = a[12];
    b.cr1 = r[0]; b.cr2 = r[1]; b.cr3 = r[2]; b.cs1 = r[3]; b.cs2 = r[4]; b.cs3 = r[5];
    b.d_s = r[6]; b.d_i = r[7]; b.pmin.x = r[8]; b.pmin.y = r[9]; b.pmin.z = r[10];
    AddIBMNode(&U->ibmlist[0], b);
  }
  return 0;
}

/* ibm_interpolation_advanced (ibm_iso.c:2572) on the current Q/lQ/P/lP. */
int ref_ibm_interpolate(int add_dundt) {
  if (!U || !IBM) return 1;
  U->ti = g_ti;
  return ibm_interpolation_advanced(U, IBM, 0, add_dundt);
}

/* FormBCS(user, alfa) (rhs.c:477) on the current Q from lQ. */
int ref_formbcs(double alfa) {
  if (!U) return 1;
  return FormBCS(U, alfa);
}

#ifdef CHIMERA_REF_WITH_MAIN
/* ---- checkpoint files through the reference's own main.c ---- */
PetscErrorCode Q_P_Binary_Output(UserCtx *user);
PetscErrorCode RestartApplication(UserCtx *user, IBMNodes *ibm, FSInfo *fsi, Cstart *cstart, PetscInt tistart);

/* Q_P_Binary_Output (main.c:247-304) of the current state as time step ti,
 * block 0, into the working directory. */
int ref_write_checkpoint(int ti) {
  if (!U) return 1;
  U->ti = ti;
  U->_this = 0;
  return Q_P_Binary_Output(U);
}

/* RestartApplication (main.c:620-693) from the files of time step ti in the
 * working directory: Q, P and Nvert read back, their ghosted copies, Qold;
 * the driver's step counter continues from ti. */
int ref_restart(int ti) {
  if (!U) return 1;
  int e = RestartApplication(U, NULL, NULL, NULL, ti);
  g_ti = ti;
  return e;
}
#endif
