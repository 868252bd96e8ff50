/*
 * chimera_b200.h -- C-ABI of libchimera_b200.so, the B200 (sm_100a) drop-in for
 * the compressible right-hand side and SSP-RK time advance of
 * madvait/Chimera_Comp_LES.
 *
 * The reference's host code keeps its PETSc vectors; it hands this library
 * plain pointers to the arrays behind them (VecGetArray of the GLOBAL Vecs on
 * one rank: AoS, natural k-j-i order, i fastest) and sizes.  State, metrics,
 * nvert mask and eddy viscosity stay resident on the GPU between calls.
 *
 * Conventions
 *   - Node counts mx,my,mz include the boundary nodes 0 and m-1, exactly as the
 *     reference's DMDA (init.c:206-218).  A periodic direction with N unique
 *     points has m = N+2 nodes (node 0 images node m-2, node m-1 images node 1).
 *   - Q is 5 doubles per node (rho, rhoU, rhoV, rhoW, rhoE) -- CompVars,
 *     variables.h:22-24.  Metrics are 3 doubles per node (Cmpnts).
 *   - Every function returns 0 on success or a CB_E* code; cb_last_error()
 *     gives a one-line message.  Calls on one context are stream-ordered and
 *     not thread-safe (one context per host thread, as the reference runs one
 *     rank per process).
 *   - No function allocates device memory except cb_create, cb_rhs (first
 *     call: its output planes), the first asynchronous transfer call
 *     (staging buffers), cb_capture_graph (graph instantiation),
 *     cb_ibm_set_surface and cb_ibm_set_list (immersed-body arrays) and,
 *     in the batched form, cb_batch_create, cb_batch_set_halo_map and
 *     cb_batch_autotune (item lists, maps, graphs).
 */
#ifndef CHIMERA_B200_H
#define CHIMERA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CB_ABI_VERSION 2

/* status codes */
#define CB_OK 0
#define CB_E_ARG 1          /* invalid argument / unsupported option combination */
#define CB_E_CUDA 2         /* CUDA runtime error (message in cb_last_error) */
#define CB_E_STATE 3        /* call out of order (e.g. step before grid/state upload) */
#define CB_E_NONFINITE 4    /* device status: NaN/Inf or rho<=0 / p<=0 seen */
#define CB_E_UNSUPPORTED 5  /* option valid in the reference but not built here */

/* precision forms */
#define CB_FP64 0   /* FP64 throughout (parity form) */
#define CB_MIXED 1  /* FP32 flux arithmetic, FP64 state / EOS / RK combine / metrics */

/* Options the reference reads from its PETSc options database on the hot
 * path; names in the comments are the reference's command-line flags. */
typedef struct {
  int mx, my, mz;       /* -im/-jm/-km (DMDA node counts) */
  int bctype[6];        /* bcs.dat: i-lo,i-hi,j-lo,j-hi,k-lo,k-hi; 7 = periodic; the face codes of
                           FormBCS (rhs.c:477-1106): i 3, 51; j 3, 10, 1; k-lo 3, 52, 55, 44, 45, 51,
                           10, 47; k-hi 3, 44, 45, 49, 51, 10, 8 */
  int les;              /* -les     : 0 off, 1 constant Smagorinsky, 2 (and every other value but 3
                           and 10) dynamic Smagorinsky with local averaging, 3 dynamic node by
                           node, 10 the LES terms without a model (nu_t stays 0); the dynamic
                           forms in single-block contexts only (Compute_Smagorinsky_Constant_1,
                           les.c:134-1472; solvers.c:28) */
  int inviscid;         /* -inv     : 1 skips formViscous */
  int fluxorder;        /* -fluxorder: 1 first order, 2 MUSCL-minmod, 3 WENO3; also the RK stage count */
  int eno_order;        /* -ENOorder: 2 or 3 */
  int central;          /* -central : 2 skew-symmetric 4-point, 3 Fp_1, other: 2-point average */
  int isothermal;       /* -isothermal */
  double s_x, s_y, s_z; /* -s_x -s_y -s_z: hybrid central weights (sensor off) */
  double ren;           /* -ren : Reynolds number */
  double ma;            /* -Ma  */
  double pr;            /* -Pr  */
  double gamma;         /* -gamma (EOS; the reference's flux code fixes 1.4) */
  double dt;            /* -dt  */
  double st;            /* Strouhal scaling of dt (init.c:98 sets 1) */
  double cs_const;      /* constant Smagorinsky coefficient (les.c:146 fixes 0.03) */
  double ci;            /* Yoshizawa constant (rhs.c:13: 0.06) */
  double ratio;         /* channel forcing ratio (0 unless channel/wavy) */
  int precision;        /* CB_FP64 or CB_MIXED */
  int device;           /* CUDA device ordinal */
  int calc_sigma;       /* -calc_sigma: pressure shock sensor for the hybrid weights (rhs.c:3333-3411) */
  double s_x_min, s_y_min, s_z_min; /* -s_x_min/-s_y_min/-s_z_min: lower bounds of the sensor (default 0) */
  double sigma_thrsh;   /* -sigma_thrsh: ks of the smoothness ratio (rhs.c:3323, default 1e-5) */
  int flux;             /* upwind flux: 0 Rusanov (the reference's, default), 1 Roe with Harten's
                           entropy fix (no counterpart in the reference) */
  double max_cs;        /* -max_cs: upper clip of the dynamic Smagorinsky coefficient (-les 2;
                           les.c:151, default 0.05) */
  double twall;         /* -Twall: wall temperature of the characteristic isothermal wall
                           (-isothermal 2 with j-wall code 1; rhs.c:486, default 1) */
  int twod;             /* -twoD: 1 is the reference's 2-D mode in i -- no i-face fluxes, a zero
                           x-momentum right-hand side, lUcat x = 0 (rhs.c:1349, 1487, 2135, 2646,
                           3168, 3465, 4215) and no x term in the characteristic wall (rhs.c:719);
                           the immersed boundary takes its own value from cb_ibm_set_options */
  int i_homo_filter, j_homo_filter, k_homo_filter;
                        /* -i/-j/-k_homo_filter: homogeneous averaging of the dynamic model's LM and
                           MM (les.c:916-1115): i alone per (k, j) line, i and k per j plane, all
                           three over the box; j or k alone only takes LM / MM node by node */
  int testfilter_ik;    /* -testfilter_ik: test-filter width 5^(1/3) instead of 2 filter widths
                           (les.c:598) */
  int visT;             /* -visT: Sutherland's law for the molecular viscosity on each face
                           (rhs.c:1412-1414, 1627-1637) */
  double tref;          /* -Tref: its reference temperature (default 273.15, rhs.c:1410) */
  int abc;              /* -ABC: with -calc_sigma, the raw sensor weights are 0 above plane
                           k = ABC (an absorbing layer; rhs.c:3311, 3341-3368); 0 off */
  int weno_order;       /* 3 (default): the reference's WENO3 with fluxorder 3; 5: WENO5-JS (Jiang & Shu,
                           J. Comput. Phys. 126 (1996)) on every face whose six-node stencil lies on the
                           nodes 0 .. m-1 and holds no wall node, the reference's path elsewhere, and no
                           (j < 30 && k < 7) MUSCL override; needs fluxorder 3.  No counterpart in the
                           reference.  Single-block contexts. */
} cb_config;

/* Fills *cfg with the reference's defaults (init.c:45-103, main.c:14-75). */
void cb_config_default(cb_config *cfg, int mx, int my, int mz);

typedef struct cb_ctx cb_ctx;

/* Creates a context and allocates the resident device arrays.
 * Replaces the vector set-up of MG_Initial (init.c:956-1090). */
int cb_create(const cb_config *cfg, cb_ctx **out);
void cb_destroy(cb_ctx *ctx);

/* Node coordinates (3 doubles per node, AoS) -> metrics on the device.
 * Replaces FormMetrics (metrics.c:3-782). */
int cb_set_grid(cb_ctx *ctx, const double *coor);

/* Host-computed metrics instead (lCsi/lEta/lZet: 3 doubles per node, lAj: 1),
 * global (unghosted) natural order. */
int cb_set_metrics(cb_ctx *ctx, const double *csi, const double *eta, const double *zet, const double *aj);

/* Metrics currently resident (lCsi/lEta/lZet 3 per node, lAj 1 per node),
 * global natural order -- what FormMetrics left in the reference's vectors. */
int cb_get_metrics(cb_ctx *ctx, double *csi, double *eta, double *zet, double *aj);

/* IBM mask, 1 double per node (Nvert, variables.h:191).  Re-upload only when
 * the body moves (ibm_search_advanced, ibm_iso.c:87). */
int cb_set_nvert(cb_ctx *ctx, const double *nvert);

/* Conserved state Q (5 doubles per node).  Sets Q and Qold, as the tail of
 * SetInitialCondition does (rhs.c:420-433); the eddy viscosity and the
 * velocity field of the last CalcUCat are reset to zero. */
int cb_upload_state(cb_ctx *ctx, const double *q);

/* Copies Q (5 per node) and, if p != NULL, the EOS pressure (1 per node) back.
 * Replaces reading user->Q / user->P after RungeKutta. */
int cb_download_state(cb_ctx *ctx, double *q, double *p);

/* Streaming host transfers, for a host that hands every step its input state
 * and takes every step's result (the reference's VecGetArray buffers, pinned
 * for the copies to overlap).  cb_upload_state_async is cb_upload_state, and
 * cb_download_state_async the Q part of cb_download_state, but each returns
 * after enqueueing: the host-to-device copy runs on an upload copy stream and
 * the device-to-host copy on a download copy stream, each through two staging
 * buffers, so the download of one step's result, the upload of the next
 * step's input and the steps themselves overlap.  The state update and the
 * packing stay ordered on the context's stream with every other call.  The
 * host may reuse an input buffer, and read an output buffer, only after
 * cb_join_transfers and cb_sync.  The first call allocates the copy streams
 * and four staging buffers (5 doubles per node each).  No counterpart in the
 * reference (its state never leaves the host). */
int cb_upload_state_async(cb_ctx *ctx, const double *q);
int cb_download_state_async(cb_ctx *ctx, double *q);
/* Orders the context's stream after every transfer enqueued so far (no host
 * wait): work or events enqueued afterwards follow the last copy. */
int cb_join_transfers(cb_ctx *ctx);

/* formRHS(user, Rhs, istage) (rhs.c:4703) on the current state: writes Rhs,
 * 5 doubles per node, zero on boundary nodes.  In LES mode the current eddy
 * viscosity is used (see cb_eddy_viscosity). */
int cb_rhs(cb_ctx *ctx, int istage, double *rhs);

/* CalcUCat (rhs.c:1322): records the current state as the velocity source of
 * the next eddy-viscosity evaluation. */
int cb_calc_ucat(cb_ctx *ctx);

/* Compute_Smagorinsky_Constant_1 + Compute_eddy_viscosity_LES
 * (les.c:135-1472, 1477-1661) from the recorded velocity field and, with
 * -les 2, the dynamic model on the current state. */
int cb_eddy_viscosity(cb_ctx *ctx);

/* Eddy viscosity Nu_t (1 double per node, global order). */
int cb_get_nut(cb_ctx *ctx, double *nut);

/* The dynamic model's coefficient user->CS (1 double per node, global order;
 * -les 2 only). */
int cb_get_cs(cb_ctx *ctx, double *cs);

/* nsteps physical time steps: per step Flow_Solver (solvers.c:13-64: LES
 * eddy viscosity, then RungeKutta solvers.c:223-294 with FormBCS and
 * EqOfState per stage) and the Q -> Qold copy of main.c:971.  Asynchronous on
 * the context's stream; returns after enqueueing. */
int cb_rk_step(cb_ctx *ctx, int nsteps);

/* Time step from the CFL condition on the current state: dt = cfl / lambda_max,
 * lambda = aj * sum_d (|m_d . u| + c |m_d|) the largest inviscid spectral radius
 * over interior fluid nodes (warp-shuffle max reduction on the device).  No
 * counterpart in the reference, which runs a fixed -dt (init.c:94); its
 * Spectral (rhs.c:4739) is an unused incompressible estimate.  Does not change
 * the context's dt; synchronises. */
int cb_cfl_dt(cb_ctx *ctx, double cfl, double *dt, double *lambda_max);

/* Autotuner of the stage kernel's k-chunk (planes per thread block along k):
 * times one stage launch per candidate on the current state (ncand = 0: every
 * k-chunk from 4 to mz-2 that changes the chunk count, then 0) and keeps the
 * fastest.  k-chunk 0 is the balanced-segment shape: one CTA per resident slot,
 * each marching an equal share of the tile columns' planes laid end to end; it
 * is kept only when 3 % faster than the best chunked grid (it moves more DRAM
 * bytes).
 * ms_out/nout (optional): per-candidate milliseconds (*nout in: capacity,
 * out: candidates timed).  Does not advance the state.  No counterpart in the
 * reference (CPU loops have no launch shape). */
int cb_autotune(cb_ctx *ctx, int ncand, const int *cand, double *ms_out, int *nout, int *best_kchunk);

/* ---- immersed boundary (ibm_interpolation_advanced, ibm_iso.c:2572-2880) ----
 *
 * The reference's host search (ibm_search_advanced, ibm_iso.c:87) stays on
 * the host: it sets nvert (pass it with cb_set_nvert) and builds one
 * interpolation list per body (user->ibmlist[ibi]).  Hand each list and the
 * body's surface to the context; every cb_rk_step then runs, after the RK
 * stages, the interpolation of each body in order (Add_dUndt = 1) and
 * FormBCS(user, 0), as RungeKutta does when -imm is set
 * (solvers.c:282-288), without a host round trip.
 *
 * One list entry: the IBMInfo fields the interpolation reads
 * (variables.h:50-89), same layout as the oracle's cbo_ibm_info. */
typedef struct {
  int ni, nj, nk;           /* the interface node (natural indices, 0 <= n < m) */
  int cell;                 /* surface element of the interception point, -1: none */
  int i1, j1, k1, i2, j2, k2, i3, j3, k3; /* donor nodes */
  int pad;                  /* unused (aligns the doubles) */
  double cr1, cr2, cr3;     /* donor weights */
  double cs1, cs2, cs3;     /* weights of the element's vertices at the interception point */
  double d_s, d_i;          /* node -> surface and surface -> donor point distances */
  double pmin[3];           /* interception point */
} cb_ibm_info;

#define CB_IBM_MAX_BODIES 16

/* IBMNodes of body ibi (variables.h:91-118): triangles nv1..nv3 (vertex
 * indices) and unit normals nf_x..nf_z of each of the n_elmt elements;
 * vertex velocities start at zero (ibm_read_ucd, ibm_io.c:1643-1653).
 * Replaces the body's surface and drops its list.  Allocates. */
int cb_ibm_set_surface(cb_ctx *ctx, int ibi, int n_v, int n_elmt, const int *nv1, const int *nv2, const int *nv3,
                       const double *nf_x, const double *nf_y, const double *nf_z);
/* Vertex velocities ibm->u and ibm->uold (n_v x (x,y,z) each, Cmpnts). */
int cb_ibm_set_velocity(cb_ctx *ctx, int ibi, const double *u, const double *uold);
/* The interpolation list of body ibi in the order the reference walks it
 * (IBMList head first), with coor the node coordinates passed to
 * cb_set_grid.  A node listed twice keeps its last entry (the later write
 * wins in the reference).  n = 0 removes the body's list.  Allocates.
 * With -isothermal 2 (the characteristic wall of ibm_iso.c:2744-2786) each
 * sweep also walks the list in order on one block for the pressure Pa that
 * the reference carries from entry to entry. */
int cb_ibm_set_list(cb_ctx *ctx, int ibi, int n, const cb_ibm_info *list, const double *coor);
/* Entries of body ibi's list after duplicate nodes were dropped (with
 * -isothermal 2 every entry is kept: its characteristic wall links each entry
 * to the one before it, and a node listed twice is written by its later
 * entry). */
int cb_ibm_count(const cb_ctx *ctx, int ibi);
/* -twoD (0, or 1/2/3: drop x/y/z from the normal and the velocity) and
 * -wallfunction (ibm_iso.c:2708-2728): 0 noslip unless -inv (then freeslip),
 * 2 the hydset log law of the wall with roughness 1e-16 (wall_function_loglaw,
 * wallfunction.c:376-420; Newton's method for u_tau), 3 freeslip.  1 returns
 * CB_E_UNSUPPORTED: the reference's Cabot wall function reads a table that
 * pre_integrate leaves in a dead stack frame (wallfunction.c:113-145). */
int cb_ibm_set_options(cb_ctx *ctx, int twoD, int wallfunction);
/* u_tau of every entry of body ibi's list (cb_ibm_count doubles, list order)
 * from the last sweep with -wallfunction 2: the values the reference keeps in
 * user->lUstar at the interface nodes (ibm_iso.c:2714-2719); 0 before. */
int cb_ibm_get_ustar(cb_ctx *ctx, int ibi, double *ustar);
/* One call of ibm_interpolation_advanced(user, ibm, ibi, Add_dUndt) on the
 * current state: five sweeps, each ending with the ghost update. */
int cb_ibm_interpolate(cb_ctx *ctx, int ibi, int add_dundt);

/* Waits for the context's stream and checks the device status word
 * (CB_E_NONFINITE when a NaN/Inf or non-positive rho/p was produced). */
int cb_sync(cb_ctx *ctx);

/* Captures one full time step into a CUDA graph; later cb_rk_step calls
 * replay it.  Returns CB_E_STATE if the state/grid are not set. */
int cb_capture_graph(cb_ctx *ctx);

/* The CUDA stream all work of this context is enqueued on (cudaStream_t). */
void *cb_stream(cb_ctx *ctx);

/* Per-kernel timing with CUDA events on the context stream (0: off, 1: on).
 * cb_timing_read returns the summed milliseconds and launch count of the
 * fused RHS/stage kernel since it was enabled, and of the whole step. */
int cb_timing_enable(cb_ctx *ctx, int on);
int cb_timing_read(cb_ctx *ctx, double *rhs_ms, int *rhs_launches, double *other_ms, int *other_launches);

/* Number of interior nodes ((mx-2)(my-2)(mz-2)) and RK stages per step. */
long long cb_interior_nodes(const cb_ctx *ctx);
int cb_stages(const cb_ctx *ctx);

/* Kernel launches one cb_rk_step(ctx, 1) enqueues. */
int cb_launches_per_step(const cb_ctx *ctx);

const char *cb_last_error(const cb_ctx *ctx);
int cb_abi_version(void);

/* Index user->ti of the last completed time step (0 after cb_create): the
 * next cb_rk_step runs step ti + 1, as the time loop of main.c:887-974 and
 * RestartApplication with tistart = ti (main.c:620) do.  Only the k-lo inflow
 * code 47 (rhs.c:904-950) reads it. */
int cb_set_time_index(cb_ctx *ctx, int ti);

/* Arithmetic-pipe peaks of GPU `device` in TFLOP/s (2 flops per fused
 * multiply-add), measured by a dependent-FMA kernel over every SM: the
 * ceiling of the compute roofline of the stage kernels.  A measurement
 * helper with no counterpart in the reference.  Allocates a small buffer,
 * synchronises. */
int cb_pipe_peaks(int device, double *fp64_tflops, double *fp32_tflops);

/* formRHS without any device allocation, for callers that may not call
 * cudaMalloc (a solver running inside a memory pool owned by another
 * framework, or a host that forbids device allocation after start-up).
 * No counterpart in the reference: there every call allocates its
 * temporaries with VecDuplicate.
 *
 * The caller owns every input and the output, all device pointers in natural
 * AoS order: d_coor 3 doubles per node, d_q 5, d_nvert 1, d_nut 1 (NULL: zero
 * eddy viscosity), d_rhs 5 (written: the RHS of formRHS at istage 0, zero on
 * boundary nodes).  Work is enqueued on `stream` (a cudaStream_t, NULL for the
 * default stream); the caller synchronises.
 *
 * Scratch lives in a file-scope __device__ array sized for
 * CB_NOALLOC_MAX_PLANE padded nodes per field, (mx+4 rounded up to 16) *
 * (my+4) * (mz+4); larger grids are rejected with CB_E_ARG.  A GPU holds the
 * array (about 20 MB) from the time the library's device module is loaded
 * there (first kernel use under CUDA's default lazy loading, start-up with
 * CUDA_MODULE_LOADING=EAGER) until the process exits.  All calls share it and
 * it keeps the last call's contents, so calls that overlap on the GPU race:
 * serialise them.  Every call looks the array's address up on the current
 * device (cudaGetSymbolAddress, no allocation); the first call on a device
 * also sets the kernels' shared-memory attributes: make it before any stream
 * capture.  Only fully periodic blocks are accepted. */
#define CB_NOALLOC_MAX_PLANE 98304LL
int cb_rhs_noalloc(const cb_config *cfg, const double *d_coor, const double *d_q, const double *d_nvert,
                   const double *d_nut, double *d_rhs, void *stream);

/* ---------------------------------------------------------------------------
 * Batched multi-block form.  Replaces the per-block loop of the reference's
 * time step (solvers.c:246, `for (bi = 0; bi < block_number; bi++)` around
 * RungeKutta) with one context holding every block resident on the GPU.
 * Per RK stage: ONE persistent stage launch whose CTAs take (block, tile,
 * k-chunk) work items, largest first, from a device counter, then one
 * on-device gather that fills every block's boundary and ghost nodes from a
 * halo map.  A whole step runs as a CUDA graph.  Blocks share the cb_config
 * (its bctype is ignored); their sizes may differ.  By default every block
 * face is an interface filled by the halo map; cb_batch_set_bctype gives a
 * block its own face codes instead.  With les and calc_sigma every block computes the
 * shock sensor's weights from its own arrays at the first stage of a step,
 * each pass followed by the wrap map (a batch with a cross-process exchange
 * refuses the sensor with CB_E_UNSUPPORTED).  With a dynamic -les (2, 3, not
 * 10) every block computes its Smagorinsky coefficient from its own arrays
 * and ghost layers once per step, as each block of the reference does on its
 * own DMDA (les.c:151-1472); -les 10 keeps nu_t zero, as in a cb_ctx.
 *
 * Per block k: cb_batch_set_grid (coordinates, 3 per node, AoS, as
 * cb_set_grid), cb_batch_set_nvert (optional; default 0), cb_batch_upload_state
 * (5 per node).  Then a halo map (cb_batch_halo_periodic for independent
 * periodic blocks, each of which then evolves exactly as it would alone in a
 * cb_ctx), cb_batch_rk_step, cb_batch_sync, cb_batch_download_state. */
typedef struct cb_batch cb_batch;
/* dims: 3 ints (mx, my, mz) per block, each >= 6 */
int cb_batch_create(const cb_config *cfg, int nblocks, const int *dims, cb_batch **out);
void cb_batch_destroy(cb_batch *b);
const char *cb_batch_last_error(const cb_batch *b);
long long cb_batch_interior_nodes(const cb_batch *b);
void *cb_batch_stream(cb_batch *b);
int cb_batch_work_items(const cb_batch *b);
int cb_batch_set_grid(cb_batch *b, int block, const double *coor);
int cb_batch_set_nvert(cb_batch *b, int block, const double *nvert);
/* Face codes of one block (6 ints: i-lo, i-hi, j-lo, j-hi, k-lo, k-hi, the
 * codes of cb_config.bctype), replacing the reference's per-block bcs.dat line
 * (init.c:556-559) and that block's FormBCS inside RungeKutta (solvers.c:246-273,
 * rhs.c:477-1227).  With a code other than 7 on any face the block runs the
 * single-block context's FormBCS on its own arrays after every stage (code 7
 * on both faces of a direction wraps the block onto itself), so it evolves
 * exactly as a cb_ctx with the same codes; it may then hold no halo-map
 * destination (set codes before the halo maps; cb_batch_halo_periodic skips
 * such blocks) and the batch takes no cross-process exchange.  Six codes 7
 * make it an interface block again.  The k-lo inflow codes 52 and 47 read
 * the node coordinates, which the block keeps from cb_batch_set_grid: give
 * them before the grid (CB_E_STATE after it); code 47's step index comes from
 * cb_batch_set_time_index, as cb_set_time_index.  CB_E_UNSUPPORTED for a
 * direction with 7 on one face only; CB_E_ARG if the block already holds a
 * halo-map destination. */
int cb_batch_set_bctype(cb_batch *b, int block, const int *bctype);
int cb_batch_set_time_index(cb_batch *b, int ti);
/* Immersed bodies in the batched form: after a block's stages the reference
 * interpolates every body on that block (ibm_interpolation_advanced with its
 * IBMList of the block), then runs FormBCS(user, 0) (solvers.c:279-288).
 * Surfaces, vertex velocities and the options are shared by all blocks (the
 * reference's ibm[ibi]; arguments as cb_ibm_set_surface / _velocity /
 * _options); each block takes its own list of each body, built as by
 * cb_ibm_set_list from that block's node coordinates.  Lists go only to
 * blocks with face codes (cb_batch_set_bctype; CB_E_UNSUPPORTED otherwise;
 * such a block then keeps face codes and its periodic directions,
 * CB_E_STATE).  A block with lists
 * advances as a cb_ctx with the same lists; its first stage reads the
 * pressure carried from its interpolation (after an upload: the EqOfState of
 * the state).  A batch with lists refuses the phase API (CB_E_UNSUPPORTED). */
int cb_batch_ibm_set_surface(cb_batch *b, int ibi, int n_v, int n_elmt, const int *nv1, const int *nv2,
                             const int *nv3, const double *nf_x, const double *nf_y, const double *nf_z);
int cb_batch_ibm_set_velocity(cb_batch *b, int ibi, const double *u, const double *uold);
int cb_batch_ibm_set_list(cb_batch *b, int block, int ibi, int n, const cb_ibm_info *list, const double *coor);
int cb_batch_ibm_set_options(cb_batch *b, int twoD, int wallfunction);
int cb_batch_upload_state(cb_batch *b, int block, const double *q);
int cb_batch_download_state(cb_batch *b, int block, double *q);
/* CFL time step over all blocks: dt = cfl / (largest spectral radius of any
 * block, as cb_cfl_dt computes it per block).  No reference counterpart (the
 * reference steps with the fixed -dt, init.c:94); the multi-process form
 * reduces lambda_max across ranks (chimera_comp_les_b200.sharded.cfl_dt). */
int cb_batch_cfl_dt(cb_batch *b, double cfl, double *dt, double *lambda_max);
/* metrics of a block as resident (csi, eta, zet 3 per node, aj 1), AoS */
int cb_batch_get_metrics(cb_batch *b, int block, double *csi, double *eta, double *zet, double *aj);
/* Halo maps: n entries of 9 ints (dst block, di, dj, dk, src block, si, sj,
 * sk, from_stage_input), node indices -2..m+1.  CB_HALO_STAGE runs after every
 * stage: the source is the stage output (then it must be an interior node) or,
 * with from_stage_input, the stage input (the reference's FormBCS reads the
 * not-yet-refreshed local vector, rhs.c:1107-1227).  CB_HALO_WRAP (the last
 * int ignored) is a plain copy within one buffer (DMGlobalToLocal across
 * blocks): applied to the eddy viscosity each step and once to the uploaded
 * state before the first step.  Destinations are non-interior nodes, each at
 * most once per map; wrap sources may not be destinations.  CB_E_ARG on a
 * violation. */
#define CB_HALO_STAGE 0
#define CB_HALO_WRAP 1
int cb_batch_set_halo_map(cb_batch *b, int kind, long long n, const int *entries);
int cb_batch_halo_periodic(cb_batch *b);
/* mode 0: one persistent stage launch over all blocks per stage; mode 1: one
 * stage launch per block (for comparison).  Asynchronous. */
int cb_batch_rk_step(cb_batch *b, int nsteps, int mode);
int cb_batch_sync(cb_batch *b);
/* Cross-process exchange (one process per GPU, each holding part of a
 * decomposed domain; the reference exchanges its DMDA ghosts with MPI inside
 * DMGlobalToLocal, init.c:156).  Halo entries whose source node lives in
 * another process are split into what this process sends (kind
 * CB_HALO_STAGE: 5 ints block,i,j,k,from_stage_input; CB_HALO_WRAP: 4 ints)
 * and what it receives (4 ints, destination nodes).  d_send / d_recv are
 * caller-owned device buffers of 5 doubles per entry, packed entry-major.
 * With an exchange the batch steps through phases: cb_batch_phase enqueues
 * the local work and packs d_send; the caller moves the buffers between
 * processes (e.g. NCCL send/recv) ordered on cb_batch_stream; then
 * cb_batch_phase_unpack scatters d_recv.  Per step: CB_PHASE_NUT (LES only),
 * then CB_PHASE_STAGE for stages 0..fluxorder-1; once after the uploads
 * CB_PHASE_STATE.  cb_batch_rk_step refuses such a batch (CB_E_STATE). */
#define CB_PHASE_STATE 0
#define CB_PHASE_NUT 1
#define CB_PHASE_STAGE 2
int cb_batch_set_exchange(cb_batch *b, int kind, long long nsend, const int *send, double *d_send, long long nrecv,
                          const int *recv, double *d_recv);
int cb_batch_phase(cb_batch *b, int phase, int stage, int mode);
int cb_batch_phase_unpack(cb_batch *b, int phase);
/* Times one persistent stage launch per candidate k-chunk of the work items
 * and keeps the fastest.  The state is not advanced. */
int cb_batch_autotune(cb_batch *b, int *best_kchunk, double *best_ms);

#ifdef __cplusplus
}
#endif
#endif
