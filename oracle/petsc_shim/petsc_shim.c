/*
 * Serial implementation of the PETSc 3.12 / MPI subset declared in
 * include/petscshim.h.  TEST INFRASTRUCTURE ONLY (see the header).
 *
 * Behaviour that the reference's hot path depends on, per PETSc's
 * documented one-rank semantics:
 *   - DMGlobalToLocal fills ghost layers of periodic directions by
 *     wrap-around (local index -1 -> global M-1, -2 -> M-2, M -> 0, ...),
 *     with box-stencil corners wrapped in every periodic direction.
 *   - DMLocalToLocal refreshes the ghosts of the destination from the
 *     owned values of the source.
 *   - VecDuplicate returns a zero-filled vector.
 */
#include "petscshim.h"
#include <stdarg.h>
#include <sys/time.h>
#include <stddef.h>

/* ------------------------------------------------------------------ */
/* options database                                                    */
/* ------------------------------------------------------------------ */
#define SHIM_MAX_OPTS 128
static char opt_name[SHIM_MAX_OPTS][64];
static char opt_val[SHIM_MAX_OPTS][64];
static int opt_n = 0;

void shim_options_clear(void) { opt_n = 0; }

int shim_options_set(const char *name, const char *value) {
  for (int i = 0; i < opt_n; i++)
    if (!strcmp(opt_name[i], name)) {
      snprintf(opt_val[i], 64, "%s", value ? value : "");
      return 0;
    }
  if (opt_n >= SHIM_MAX_OPTS) return 1;
  snprintf(opt_name[opt_n], 64, "%s", name);
  snprintf(opt_val[opt_n], 64, "%s", value ? value : "");
  opt_n++;
  return 0;
}

static const char *opt_find(const char *name) {
  for (int i = 0; i < opt_n; i++)
    if (!strcmp(opt_name[i], name)) return opt_val[i];
  return NULL;
}

PetscErrorCode PetscOptionsGetInt(void *o, const char *pre, const char *name, PetscInt *v, PetscBool *set) {
  (void)o; (void)pre;
  const char *s = opt_find(name);
  if (s) { *v = (PetscInt)strtol(s, NULL, 10); }
  if (set) *set = s ? PETSC_TRUE : PETSC_FALSE;
  return 0;
}

PetscErrorCode PetscOptionsGetReal(void *o, const char *pre, const char *name, PetscReal *v, PetscBool *set) {
  (void)o; (void)pre;
  const char *s = opt_find(name);
  if (s) { *v = strtod(s, NULL); }
  if (set) *set = s ? PETSC_TRUE : PETSC_FALSE;
  return 0;
}

PetscErrorCode PetscOptionsGetIntArray(void *o, const char *pre, const char *name, PetscInt *v, PetscInt *n, PetscBool *set) {
  (void)o; (void)pre;
  const char *s = opt_find(name);
  int cnt = 0;
  if (s) {
    const char *p = s;
    while (*p && cnt < *n) {
      char *end;
      long x = strtol(p, &end, 10);
      if (end == p) break;
      v[cnt++] = (PetscInt)x;
      p = end;
      while (*p == ',' || *p == ' ') p++;
    }
    *n = cnt;
  }
  if (set) *set = s ? PETSC_TRUE : PETSC_FALSE;
  return 0;
}

PetscErrorCode PetscOptionsGetRealArray(void *o, const char *pre, const char *name, PetscReal *v, PetscInt *n, PetscBool *set) {
  (void)o; (void)pre;
  const char *s = opt_find(name);
  int cnt = 0;
  if (s) {
    const char *p = s;
    while (*p && cnt < *n) {
      char *end;
      double x = strtod(p, &end);
      if (end == p) break;
      v[cnt++] = x;
      p = end;
      while (*p == ',' || *p == ' ') p++;
    }
    *n = cnt;
  }
  if (set) *set = s ? PETSC_TRUE : PETSC_FALSE;
  return 0;
}

PetscErrorCode PetscOptionsHasName(void *o, const char *pre, const char *name, PetscBool *set) {
  (void)o; (void)pre;
  if (set) *set = opt_find(name) ? PETSC_TRUE : PETSC_FALSE;
  return 0;
}

PetscErrorCode PetscOptionsGetString(void *o, const char *pre, const char *name, char *v, size_t len, PetscBool *set) {
  (void)o; (void)pre;
  const char *s = opt_find(name);
  if (s && len) snprintf(v, len, "%s", s);
  if (set) *set = s ? PETSC_TRUE : PETSC_FALSE;
  return 0;
}

PetscErrorCode PetscOptionsInsertFile(MPI_Comm c, void *o, const char *f, PetscBool r) {
  (void)c; (void)o; (void)f; (void)r;
  return 0;
}

/* ------------------------------------------------------------------ */
/* printing / misc                                                     */
/* ------------------------------------------------------------------ */
static int shim_verbose(void) {
  static int v = -1;
  if (v < 0) { const char *e = getenv("CHIMERA_SHIM_VERBOSE"); v = (e && *e == '1'); }
  return v;
}

PetscErrorCode PetscPrintf(MPI_Comm c, const char *fmt, ...) {
  (void)c;
  if (shim_verbose()) { va_list ap; va_start(ap, fmt); vfprintf(stderr, fmt, ap); va_end(ap); }
  return 0;
}
PetscErrorCode PetscFPrintf(MPI_Comm c, FILE *f, const char *fmt, ...) {
  (void)c;
  va_list ap; va_start(ap, fmt); vfprintf(f ? f : stderr, fmt, ap); va_end(ap);
  return 0;
}
PetscErrorCode PetscSynchronizedPrintf(MPI_Comm c, const char *fmt, ...) {
  (void)c;
  if (shim_verbose()) { va_list ap; va_start(ap, fmt); vfprintf(stderr, fmt, ap); va_end(ap); }
  return 0;
}
PetscErrorCode PetscSynchronizedFlush(MPI_Comm c, FILE *f) { (void)c; (void)f; return 0; }
PetscErrorCode PetscBarrier(void *o) { (void)o; return 0; }
PetscErrorCode PetscTime(PetscLogDouble *t) {
  struct timeval tv; gettimeofday(&tv, NULL);
  *t = tv.tv_sec + 1e-6 * tv.tv_usec;
  return 0;
}
PetscErrorCode PetscGetTime(PetscLogDouble *t) { return PetscTime(t); }
PetscErrorCode PetscMalloc(size_t n, void *p) { *(void **)p = calloc(1, n ? n : 1); return 0; }
PetscErrorCode PetscFree(void *p) { free(p); return 0; }
PetscErrorCode PetscGlobalMax(MPI_Comm c, const PetscReal *l, PetscReal *g) { (void)c; *g = *l; return 0; }
PetscErrorCode PetscGlobalMin(MPI_Comm c, const PetscReal *l, PetscReal *g) { (void)c; *g = *l; return 0; }
PetscErrorCode PetscGlobalSum(MPI_Comm c, const PetscReal *l, PetscReal *g) { (void)c; *g = *l; return 0; }

/* ------------------------------------------------------------------ */
/* MPI, one rank: every reduction is the identity                     */
/* ------------------------------------------------------------------ */
static size_t mpi_size(MPI_Datatype t) {
  switch (t) { case MPI_DOUBLE: return sizeof(double); case MPI_INT: return sizeof(int);
               case MPI_FLOAT: return sizeof(float); default: return 1; }
}
int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  (void)op; (void)c;
  if (s != r) memmove(r, s, (size_t)count * mpi_size(t));
  return 0;
}
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c) {
  (void)root;
  return MPI_Allreduce(s, r, count, t, op, c);
}
int MPI_Bcast(void *b, int count, MPI_Datatype t, int root, MPI_Comm c) { (void)b; (void)count; (void)t; (void)root; (void)c; return 0; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

/* ------------------------------------------------------------------ */
/* DMDA geometry helpers                                               */
/* ------------------------------------------------------------------ */
static void dm_ghost_range(DM dm, int dir, PetscInt *gs, PetscInt *gm) {
  PetscInt M = dir == 0 ? dm->M : dir == 1 ? dm->N : dm->P;
  DMBoundaryType b = dir == 0 ? dm->bx : dir == 1 ? dm->by : dm->bz;
  if (b == DM_BOUNDARY_PERIODIC || b == DM_BOUNDARY_GHOSTED) { *gs = -dm->s; *gm = M + 2 * dm->s; }
  else { *gs = 0; *gm = M; }
}

static PetscInt dm_local_n(DM dm) {
  PetscInt gs, gx, gy, gz;
  dm_ghost_range(dm, 0, &gs, &gx);
  dm_ghost_range(dm, 1, &gs, &gy);
  dm_ghost_range(dm, 2, &gs, &gz);
  return gx * gy * gz * dm->dof;
}

static Vec vec_new(PetscInt n, DM dm, int local) {
  Vec v = (Vec)calloc(1, sizeof(struct _p_Vec));
  v->a = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  v->n = n;
  v->dm = dm;
  v->local = local;
  return v;
}

/* ------------------------------------------------------------------ */
/* Vec                                                                 */
/* ------------------------------------------------------------------ */
PetscErrorCode VecDuplicate(Vec v, Vec *out) { *out = vec_new(v->n, v->dm, v->local); return 0; }

PetscErrorCode VecDestroy(Vec *v) {
  if (!v || !*v) return 0;
  free((*v)->a);
  free((*v)->arr_k);
  free((*v)->arr_j);
  free(*v);
  *v = NULL;
  return 0;
}

PetscErrorCode VecSet(Vec v, PetscScalar a) { for (PetscInt i = 0; i < v->n; i++) v->a[i] = a; return 0; }
PetscErrorCode VecCopy(Vec x, Vec y) { if (x != y) memcpy(y->a, x->a, sizeof(double) * (size_t)x->n); return 0; }

PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y) {
  for (PetscInt i = 0; i < w->n; i++) w->a[i] = y->a[i] + a * x->a[i];
  return 0;
}
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x) { for (PetscInt i = 0; i < y->n; i++) y->a[i] += a * x->a[i]; return 0; }
PetscErrorCode VecAYPX(Vec y, PetscScalar b, Vec x) { for (PetscInt i = 0; i < y->n; i++) y->a[i] = x->a[i] + b * y->a[i]; return 0; }
PetscErrorCode VecAXPBY(Vec y, PetscScalar a, PetscScalar b, Vec x) {
  for (PetscInt i = 0; i < y->n; i++) y->a[i] = a * x->a[i] + b * y->a[i];
  return 0;
}
PetscErrorCode VecAXPBYPCZ(Vec z, PetscScalar a, PetscScalar b, PetscScalar c, Vec x, Vec y) {
  for (PetscInt i = 0; i < z->n; i++) z->a[i] = a * x->a[i] + b * y->a[i] + c * z->a[i];
  return 0;
}
PetscErrorCode VecScale(Vec x, PetscScalar a) { for (PetscInt i = 0; i < x->n; i++) x->a[i] *= a; return 0; }
PetscErrorCode VecShift(Vec x, PetscScalar a) { for (PetscInt i = 0; i < x->n; i++) x->a[i] += a; return 0; }
PetscErrorCode VecPointwiseMult(Vec w, Vec x, Vec y) { for (PetscInt i = 0; i < w->n; i++) w->a[i] = x->a[i] * y->a[i]; return 0; }

PetscErrorCode VecNorm(Vec x, NormType t, PetscReal *r) {
  double s = 0.0;
  for (PetscInt i = 0; i < x->n; i++) {
    double v = fabs(x->a[i]);
    if (t == NORM_INFINITY) { if (v > s) s = v; }
    else if (t == NORM_1) s += v;
    else s += v * v;
  }
  *r = (t == NORM_2 || t == NORM_FROBENIUS) ? sqrt(s) : s;
  return 0;
}
PetscErrorCode VecMax(Vec x, PetscInt *idx, PetscReal *r) {
  double m = -INFINITY; PetscInt k = -1;
  for (PetscInt i = 0; i < x->n; i++) if (x->a[i] > m) { m = x->a[i]; k = i; }
  if (idx) *idx = k;
  *r = m;
  return 0;
}
PetscErrorCode VecMin(Vec x, PetscInt *idx, PetscReal *r) {
  double m = INFINITY; PetscInt k = -1;
  for (PetscInt i = 0; i < x->n; i++) if (x->a[i] < m) { m = x->a[i]; k = i; }
  if (idx) *idx = k;
  *r = m;
  return 0;
}
PetscErrorCode VecSum(Vec x, PetscScalar *r) { double s = 0; for (PetscInt i = 0; i < x->n; i++) s += x->a[i]; *r = s; return 0; }
PetscErrorCode VecStrideSet(Vec v, PetscInt field, PetscScalar a) {
  PetscInt bs = v->dm ? v->dm->dof : 1;
  for (PetscInt i = field; i < v->n; i += bs) v->a[i] = a;
  return 0;
}
PetscErrorCode VecGetSize(Vec v, PetscInt *n) { *n = v->n; return 0; }
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n) { *n = v->n; return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a) { (void)v; *a = NULL; return 0; }

/* ------------------------------------------------------------------ */
/* DM                                                                  */
/* ------------------------------------------------------------------ */
PetscErrorCode DMDACreate3d(MPI_Comm c, DMBoundaryType bx, DMBoundaryType by, DMBoundaryType bz,
                            DMDAStencilType st, PetscInt M, PetscInt N, PetscInt P, PetscInt m,
                            PetscInt n, PetscInt p, PetscInt dof, PetscInt s, const PetscInt *lx,
                            const PetscInt *ly, const PetscInt *lz, DM *da) {
  (void)c; (void)m; (void)n; (void)p; (void)lx; (void)ly; (void)lz;
  DM d = (DM)calloc(1, sizeof(struct _p_DM));
  d->M = M; d->N = N; d->P = P; d->dof = dof; d->s = s;
  d->bx = bx; d->by = by; d->bz = bz; d->st = st;
  *da = d;
  return 0;
}
PetscErrorCode DMSetFromOptions(DM dm) { (void)dm; return 0; }
PetscErrorCode DMSetUp(DM dm) { (void)dm; return 0; }
PetscErrorCode DMDestroy(DM *dm) {
  if (!dm || !*dm) return 0;
  if ((*dm)->cdm) {
    VecDestroy(&(*dm)->coords);
    VecDestroy(&(*dm)->lcoords);
    free((*dm)->cdm);
  }
  free(*dm);
  *dm = NULL;
  return 0;
}

PetscErrorCode DMCreateGlobalVector(DM dm, Vec *v) { *v = vec_new(dm->M * dm->N * dm->P * dm->dof, dm, 0); return 0; }
PetscErrorCode DMCreateLocalVector(DM dm, Vec *v) { *v = vec_new(dm_local_n(dm), dm, 1); return 0; }

PetscErrorCode DMDAGetLocalInfo(DM dm, DMDALocalInfo *info) {
  memset(info, 0, sizeof(*info));
  info->dim = 3; info->dof = dm->dof; info->sw = dm->s;
  info->mx = dm->M; info->my = dm->N; info->mz = dm->P;
  info->xs = info->ys = info->zs = 0;
  info->xm = dm->M; info->ym = dm->N; info->zm = dm->P;
  dm_ghost_range(dm, 0, &info->gxs, &info->gxm);
  dm_ghost_range(dm, 1, &info->gys, &info->gym);
  dm_ghost_range(dm, 2, &info->gzs, &info->gzm);
  info->bx = dm->bx; info->by = dm->by; info->bz = dm->bz; info->st = dm->st;
  info->da = dm;
  return 0;
}

PetscErrorCode DMDAGetInfo(DM dm, PetscInt *dim, PetscInt *M, PetscInt *N, PetscInt *P, PetscInt *m,
                           PetscInt *n, PetscInt *p, PetscInt *dof, PetscInt *s, DMBoundaryType *bx,
                           DMBoundaryType *by, DMBoundaryType *bz, DMDAStencilType *st) {
  if (dim) *dim = 3;
  if (M) *M = dm->M;
  if (N) *N = dm->N;
  if (P) *P = dm->P;
  if (m) *m = 1;
  if (n) *n = 1;
  if (p) *p = 1;
  if (dof) *dof = dm->dof;
  if (s) *s = dm->s;
  if (bx) *bx = dm->bx;
  if (by) *by = dm->by;
  if (bz) *bz = dm->bz;
  if (st) *st = dm->st;
  return 0;
}

PetscErrorCode DMDAGetCorners(DM dm, PetscInt *x, PetscInt *y, PetscInt *z, PetscInt *m, PetscInt *n, PetscInt *p) {
  if (x) *x = 0;
  if (y) *y = 0;
  if (z) *z = 0;
  if (m) *m = dm->M;
  if (n) *n = dm->N;
  if (p) *p = dm->P;
  return 0;
}
PetscErrorCode DMDAGetGhostCorners(DM dm, PetscInt *x, PetscInt *y, PetscInt *z, PetscInt *m, PetscInt *n, PetscInt *p) {
  PetscInt gs, gm;
  dm_ghost_range(dm, 0, &gs, &gm); if (x) *x = gs; if (m) *m = gm;
  dm_ghost_range(dm, 1, &gs, &gm); if (y) *y = gs; if (n) *n = gm;
  dm_ghost_range(dm, 2, &gs, &gm); if (z) *z = gs; if (p) *p = gm;
  return 0;
}

/* Build (and cache on the Vec) a k->j->i pointer structure whose indices are
 * global node indices, offset by the ghost start for local vectors. */
PetscErrorCode DMDAVecGetArray(DM dm, Vec v, void *array) {
  PetscInt xs, xm, ys, ym, zs, zm;
  size_t esize = sizeof(double) * (size_t)dm->dof;
  if (v->n == dm->M * dm->N * dm->P * dm->dof && !v->local) {
    xs = ys = zs = 0; xm = dm->M; ym = dm->N; zm = dm->P;
  } else {
    dm_ghost_range(dm, 0, &xs, &xm);
    dm_ghost_range(dm, 1, &ys, &ym);
    dm_ghost_range(dm, 2, &zs, &zm);
  }
  if ((size_t)xm * ym * zm * dm->dof != (size_t)v->n) {
    fprintf(stderr, "petsc shim: DMDAVecGetArray size mismatch (vec %d, dm %d)\n", v->n, xm * ym * zm * dm->dof);
    abort();
  }
  if (!v->arr_k || v->arr_esize != (int)esize) {
    free(v->arr_k);
    free(v->arr_j);
    char ***kp = (char ***)malloc(sizeof(char **) * (size_t)zm);
    char **jp = (char **)malloc(sizeof(char *) * (size_t)zm * ym);
    for (PetscInt k = 0; k < zm; k++) {
      for (PetscInt j = 0; j < ym; j++)
        jp[(size_t)k * ym + j] = (char *)v->a + ((size_t)k * ym + j) * xm * esize - (ptrdiff_t)xs * (ptrdiff_t)esize;
      kp[k] = jp + (size_t)k * ym - ys;
    }
    v->arr_k = kp;
    v->arr_j = jp;
    v->arr_esize = (int)esize;
  }
  *(char ****)array = (char ***)v->arr_k - zs;
  return 0;
}

/* PETSc 3.12's DMDAVecRestoreArray (VecRestoreArray3d) frees the row-pointer
 * table but leaves the caller's pointer as it was; les.c:417-419 reads csi,
 * eta and zet after restoring them (les.c:400-402) and works only because the
 * freed table still holds valid rows.  The shim keeps its table alive with the
 * Vec, so leaving the pointer as it was reproduces that behaviour without a
 * use after free. */
PetscErrorCode DMDAVecRestoreArray(DM dm, Vec v, void *array) { (void)dm; (void)v; (void)array; return 0; }

static inline PetscInt wrap(PetscInt i, PetscInt M) { i %= M; return i < 0 ? i + M : i; }

/* Fill every entry of a local vector from a source array indexed by global
 * node (periodic wrap), reading owned values of `src` laid out either as a
 * global vector (src_local = 0) or a local vector (src_local = 1). */
static void fill_local(DM dm, const double *src, int src_local, double *dst) {
  PetscInt gxs, gxm, gys, gym, gzs, gzm;
  dm_ghost_range(dm, 0, &gxs, &gxm);
  dm_ghost_range(dm, 1, &gys, &gym);
  dm_ghost_range(dm, 2, &gzs, &gzm);
  PetscInt dof = dm->dof;
  for (PetscInt k = 0; k < gzm; k++) {
    PetscInt kg = wrap(k + gzs, dm->P);
    for (PetscInt j = 0; j < gym; j++) {
      PetscInt jg = wrap(j + gys, dm->N);
      for (PetscInt i = 0; i < gxm; i++) {
        PetscInt ig = wrap(i + gxs, dm->M);
        size_t sidx;
        if (src_local) sidx = ((size_t)(kg - gzs) * gym + (jg - gys)) * gxm + (ig - gxs);
        else sidx = ((size_t)kg * dm->N + jg) * dm->M + ig;
        size_t didx = ((size_t)k * gym + j) * gxm + i;
        memcpy(dst + didx * dof, src + sidx * dof, sizeof(double) * (size_t)dof);
      }
    }
  }
}

PetscErrorCode DMGlobalToLocalBegin(DM dm, Vec g, InsertMode mode, Vec l) {
  (void)mode;
  fill_local(dm, g->a, 0, l->a);
  return 0;
}
PetscErrorCode DMGlobalToLocalEnd(DM dm, Vec g, InsertMode mode, Vec l) { (void)dm; (void)g; (void)mode; (void)l; return 0; }

PetscErrorCode DMLocalToGlobalBegin(DM dm, Vec l, InsertMode mode, Vec g) {
  PetscInt gxs, gxm, gys, gym, gzs, gzm;
  dm_ghost_range(dm, 0, &gxs, &gxm);
  dm_ghost_range(dm, 1, &gys, &gym);
  dm_ghost_range(dm, 2, &gzs, &gzm);
  PetscInt dof = dm->dof;
  for (PetscInt k = 0; k < dm->P; k++)
    for (PetscInt j = 0; j < dm->N; j++)
      for (PetscInt i = 0; i < dm->M; i++) {
        size_t sidx = ((size_t)(k - gzs) * gym + (j - gys)) * gxm + (i - gxs);
        size_t didx = ((size_t)k * dm->N + j) * dm->M + i;
        for (PetscInt d = 0; d < dof; d++) {
          if (mode == ADD_VALUES) g->a[didx * dof + d] += l->a[sidx * dof + d];
          else g->a[didx * dof + d] = l->a[sidx * dof + d];
        }
      }
  return 0;
}
PetscErrorCode DMLocalToGlobalEnd(DM dm, Vec l, InsertMode mode, Vec g) { (void)dm; (void)l; (void)mode; (void)g; return 0; }

PetscErrorCode DMLocalToLocalBegin(DM dm, Vec a, InsertMode mode, Vec b) {
  (void)mode;
  if (a == b) {
    double *tmp = (double *)malloc(sizeof(double) * (size_t)a->n);
    memcpy(tmp, a->a, sizeof(double) * (size_t)a->n);
    fill_local(dm, tmp, 1, b->a);
    free(tmp);
  } else {
    fill_local(dm, a->a, 1, b->a);
  }
  return 0;
}
PetscErrorCode DMLocalToLocalEnd(DM dm, Vec a, InsertMode mode, Vec b) { (void)dm; (void)a; (void)mode; (void)b; return 0; }

static void ensure_cdm(DM dm) {
  if (dm->cdm) return;
  DM c = (DM)calloc(1, sizeof(struct _p_DM));
  *c = *dm;
  c->dof = 3;
  c->cdm = NULL;
  c->coords = c->lcoords = NULL;
  c->is_coord_dm = 1;
  dm->cdm = c;
  DMCreateGlobalVector(c, &dm->coords);
  DMCreateLocalVector(c, &dm->lcoords);
}

PetscErrorCode DMDASetUniformCoordinates(DM dm, PetscReal x0, PetscReal x1, PetscReal y0, PetscReal y1, PetscReal z0, PetscReal z1) {
  ensure_cdm(dm);
  double hx = dm->M > 1 ? (x1 - x0) / (dm->M - 1) : 0, hy = dm->N > 1 ? (y1 - y0) / (dm->N - 1) : 0,
         hz = dm->P > 1 ? (z1 - z0) / (dm->P - 1) : 0;
  for (PetscInt k = 0; k < dm->P; k++)
    for (PetscInt j = 0; j < dm->N; j++)
      for (PetscInt i = 0; i < dm->M; i++) {
        size_t id = ((size_t)k * dm->N + j) * dm->M + i;
        dm->coords->a[3 * id + 0] = x0 + hx * i;
        dm->coords->a[3 * id + 1] = y0 + hy * j;
        dm->coords->a[3 * id + 2] = z0 + hz * k;
      }
  fill_local(dm->cdm, dm->coords->a, 0, dm->lcoords->a);
  return 0;
}

PetscErrorCode DMGetCoordinateDM(DM dm, DM *cdm) { ensure_cdm(dm); *cdm = dm->cdm; return 0; }
PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec *c) {
  ensure_cdm(dm);
  fill_local(dm->cdm, dm->coords->a, 0, dm->lcoords->a);
  *c = dm->lcoords;
  return 0;
}
PetscErrorCode DMGetCoordinates(DM dm, Vec *c) { ensure_cdm(dm); *c = dm->coords; return 0; }

/* ------------------------------------------------------------------ */
/* Binary viewer: PetscViewerBinaryOpen / VecView / VecLoad in PETSc's */
/* binary Vec format -- int32 VEC_FILE_CLASSID (1211214), int32 global */
/* length, the values as big-endian float64; a DMDA Vec in natural     */
/* (k-j-i, dof-interleaved) order, which on one rank is the global     */
/* Vec's own order.  Opening a file for writing also opens its ".info" */
/* side file, to which VecView adds "-vecload_block_size <dof>" for a  */
/* Vec of more than one component (what VecLoad reads back).           */
/* ------------------------------------------------------------------ */
#define SHIM_VEC_FILE_CLASSID 1211214
struct _p_PetscViewer {
  FILE *f, *info;
  PetscFileMode mode;
};

static void put_be32(FILE *f, int v) {
  unsigned char b[4] = {(unsigned char)(v >> 24), (unsigned char)(v >> 16), (unsigned char)(v >> 8), (unsigned char)v};
  fwrite(b, 1, 4, f);
}
static int get_be32(FILE *f, int *v) {
  unsigned char b[4];
  if (fread(b, 1, 4, f) != 4) return 1;
  *v = (int)(((unsigned)b[0] << 24) | ((unsigned)b[1] << 16) | ((unsigned)b[2] << 8) | (unsigned)b[3]);
  return 0;
}

PetscErrorCode PetscViewerBinaryOpen(MPI_Comm c, const char *name, PetscFileMode mode, PetscViewer *v) {
  (void)c;
  PetscViewer w = (PetscViewer)calloc(1, sizeof(struct _p_PetscViewer));
  w->mode = mode;
  w->f = fopen(name, mode == FILE_MODE_READ ? "rb" : "wb");
  if (!w->f) { free(w); *v = NULL; return 1; }
  if (mode != FILE_MODE_READ) {
    char info[PETSC_MAX_PATH_LEN];
    snprintf(info, sizeof info, "%s.info", name);
    w->info = fopen(info, "w");
  }
  *v = w;
  return 0;
}
PetscErrorCode PetscViewerDestroy(PetscViewer *v) {
  if (!v || !*v) return 0;
  if ((*v)->f) fclose((*v)->f);
  if ((*v)->info) fclose((*v)->info);
  free(*v);
  *v = NULL;
  return 0;
}
PetscErrorCode VecView(Vec x, PetscViewer v) {
  if (!v || !v->f || v->mode == FILE_MODE_READ || x->local) return 1;
  put_be32(v->f, SHIM_VEC_FILE_CLASSID);
  put_be32(v->f, x->n);
  for (PetscInt t = 0; t < x->n; t++) {
    unsigned long long u;
    memcpy(&u, &x->a[t], 8);
    unsigned char b[8];
    for (int k = 0; k < 8; k++) b[k] = (unsigned char)(u >> (56 - 8 * k));
    fwrite(b, 1, 8, v->f);
  }
  if (v->info && x->dm && x->dm->dof > 1) fprintf(v->info, "-vecload_block_size %d\n", (int)x->dm->dof);
  return 0;
}
PetscErrorCode VecLoad(Vec x, PetscViewer v) {
  int cls = 0, n = 0;
  if (!v || !v->f || v->mode != FILE_MODE_READ || x->local) return 1;
  if (get_be32(v->f, &cls) || cls != SHIM_VEC_FILE_CLASSID || get_be32(v->f, &n) || n != x->n) return 1;
  for (PetscInt t = 0; t < x->n; t++) {
    unsigned char b[8];
    if (fread(b, 1, 8, v->f) != 8) return 1;
    unsigned long long u = 0;
    for (int k = 0; k < 8; k++) u = (u << 8) | b[k];
    memcpy(&x->a[t], &u, 8);
  }
  return 0;
}
/* VTK viewer calls of the reference's Q_P_VTK_Input (never run here) */
PetscErrorCode PetscViewerCreate(MPI_Comm c, PetscViewer *v) { (void)c; *v = (PetscViewer)calloc(1, sizeof(struct _p_PetscViewer)); return 0; }
PetscErrorCode PetscViewerSetType(PetscViewer v, const char *t) { (void)v; (void)t; return 0; }
PetscErrorCode PetscViewerFileSetMode(PetscViewer v, PetscFileMode m) { if (v) v->mode = m; return 0; }
PetscErrorCode PetscViewerFileSetName(PetscViewer v, const char *n) { (void)v; (void)n; return 1; }
PetscErrorCode PetscObjectSetName(PetscObject o, const char *n) { (void)o; (void)n; return 0; }
PetscErrorCode PetscObjectSetOptionsPrefix(PetscObject o, const char *p) { (void)o; (void)p; return 0; }
PetscErrorCode PetscOptionsClearValue(void *o, const char *n) { (void)o; (void)n; return 0; }
