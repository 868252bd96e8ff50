/*
 * Serial stand-in for the subset of PETSc 3.12 / MPI that the reference's
 * compressible hot path (rhs.c, les.c, metrics.c, solvers.c) calls.
 *
 * TEST INFRASTRUCTURE ONLY: this shim exists so that the reference's own
 * source files compile unmodified into oracle/_ref/ and can pin the oracle.
 * Nothing in the product links it.
 *
 * Semantics follow PETSc's documented API for one MPI rank:
 *   - DMDA vectors are node-based, dof-interleaved (AoS), natural k-j-i order.
 *   - A local (ghosted) vector of a periodic direction carries `s` ghost
 *     layers on each side filled by wrap-around (global index mod M).
 *     Non-periodic directions have no ghost layers outside the domain.
 *   - VecDuplicate / VecCreate zero-initialise (PETSc allocates with calloc).
 */
#ifndef PETSCSHIM_H
#define PETSCSHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscReal;
typedef double PetscScalar;
typedef double PetscLogDouble;
typedef int PetscErrorCode;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define PETSC_COMM_WORLD 0
#define PETSC_COMM_SELF 1
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_CHAR 4
#define MPIU_REAL MPI_DOUBLE
#define MPIU_SCALAR MPI_DOUBLE
#define MPIU_INT MPI_INT
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPIU_SUM MPI_SUM
#define MPIU_MAX MPI_MAX
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

#define PETSC_NULL NULL
#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_DETERMINE PETSC_DECIDE
#define PETSC_MAX_PATH_LEN 4096
#define PETSC_PI 3.14159265358979323846

/* petscmath.h definitions (PETSc 3.12) */
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
#define PetscMax(a, b) (((a) < (b)) ? (b) : (a))
#define PetscSign(a) (((a) >= 0) ? ((a) == 0 ? 0 : 1) : -1)
#define PetscAbsScalar(a) fabs(a)
#define PetscAbsReal(a) fabs(a)
#define PetscAbsInt(a) (((a) < 0) ? -(a) : (a))
#define PetscSqrtReal(a) sqrt(a)
#define PetscSqrtScalar(a) sqrt(a)
#define PetscPowReal(a, b) pow(a, b)
#define PetscPowScalar(a, b) pow(a, b)
#define PetscRealPart(a) (a)
#define PetscSqr(a) ((a) * (a))

#define CHKERRQ(e) do { if (e) return (e); } while (0)
#define CHKERRABORT(c, e) do { if (e) abort(); } while (0)
#define SETERRQ(c, n, s) return (n)
#define SETERRQ1(c, n, s, a1) return (n)
#define SETERRQ2(c, n, s, a1, a2) return (n)
#define PetscFunctionBegin
#define PetscFunctionReturn(x) return (x)

typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_FROBENIUS = 2, NORM_INFINITY = 3 } NormType;
typedef enum { DM_BOUNDARY_NONE = 0, DM_BOUNDARY_GHOSTED = 1, DM_BOUNDARY_MIRROR = 2, DM_BOUNDARY_PERIODIC = 3 } DMBoundaryType;
typedef enum { DMDA_STENCIL_STAR = 0, DMDA_STENCIL_BOX = 1 } DMDAStencilType;
typedef enum { FILE_MODE_READ = 0, FILE_MODE_WRITE = 1, FILE_MODE_APPEND = 2 } PetscFileMode;

struct _p_DM;
typedef struct _p_DM *DM;

struct _p_Vec {
  double *a;          /* data, dof-interleaved */
  PetscInt n;         /* number of doubles */
  struct _p_DM *dm;   /* owning DMDA (may be NULL) */
  int local;          /* 1: ghosted local vector */
  void *arr_k;        /* cached 3-D access arrays (DMDAVecGetArray) */
  void *arr_j;
  int arr_esize;
};
typedef struct _p_Vec *Vec;

typedef struct {
  PetscInt dim, dof, sw;
  PetscInt mx, my, mz;
  PetscInt xs, ys, zs;
  PetscInt xm, ym, zm;
  PetscInt gxs, gys, gzs;
  PetscInt gxm, gym, gzm;
  DMBoundaryType bx, by, bz;
  DMDAStencilType st;
  DM da;
} DMDALocalInfo;

struct _p_DM {
  PetscInt M, N, P, dof, s;
  DMBoundaryType bx, by, bz;
  DMDAStencilType st;
  struct _p_DM *cdm; /* coordinate DM (dof 3) */
  Vec coords;        /* global coordinates */
  Vec lcoords;       /* local (ghosted) coordinates */
  int is_coord_dm;
};

/* Opaque types named by variables.h that the hot path never dereferences. */
typedef struct _p_Mat *Mat;
typedef struct _p_KSP *KSP;
typedef struct _p_SNES *SNES;
typedef struct _p_AO *AO;
typedef struct _p_MatNullSpace *MatNullSpace;
typedef struct _p_ISColoring *ISColoring;
typedef struct _p_MatFDColoring *MatFDColoring;
typedef struct _p_PetscViewer *PetscViewer;
typedef struct _p_IS *IS;
typedef struct _p_PC *PC;
typedef struct _p_VecScatter *VecScatter;
typedef struct _p_PetscRandom *PetscRandom;

/* ---- options database (driver fills it; hot path reads it) ---- */
PetscErrorCode PetscOptionsGetInt(void *opt, const char *pre, const char *name, PetscInt *v, PetscBool *set);
PetscErrorCode PetscOptionsGetReal(void *opt, const char *pre, const char *name, PetscReal *v, PetscBool *set);
PetscErrorCode PetscOptionsGetIntArray(void *opt, const char *pre, const char *name, PetscInt *v, PetscInt *n, PetscBool *set);
PetscErrorCode PetscOptionsGetRealArray(void *opt, const char *pre, const char *name, PetscReal *v, PetscInt *n, PetscBool *set);
PetscErrorCode PetscOptionsHasName(void *opt, const char *pre, const char *name, PetscBool *set);
PetscErrorCode PetscOptionsGetString(void *opt, const char *pre, const char *name, char *v, size_t len, PetscBool *set);
PetscErrorCode PetscOptionsInsertFile(MPI_Comm c, void *opt, const char *file, PetscBool req);
void shim_options_clear(void);
int shim_options_set(const char *name, const char *value);

/* ---- printing / misc ---- */
PetscErrorCode PetscPrintf(MPI_Comm c, const char *fmt, ...);
PetscErrorCode PetscFPrintf(MPI_Comm c, FILE *f, const char *fmt, ...);
PetscErrorCode PetscSynchronizedPrintf(MPI_Comm c, const char *fmt, ...);
PetscErrorCode PetscSynchronizedFlush(MPI_Comm c, FILE *f);
PetscErrorCode PetscBarrier(void *obj);
PetscErrorCode PetscTime(PetscLogDouble *t);
PetscErrorCode PetscGetTime(PetscLogDouble *t);
PetscErrorCode PetscMalloc(size_t n, void *p);
PetscErrorCode PetscFree(void *p);
#define PetscNew(p) (*(p) = calloc(1, sizeof(**(p))), 0)
#define PetscMalloc1(n, p) (*(p) = calloc((size_t)(n) + 1, sizeof(**(p))), 0)
#define PetscCalloc1(n, p) (*(p) = calloc((size_t)(n) + 1, sizeof(**(p))), 0)
#define PetscMemzero(p, n) (memset((p), 0, (n)), 0)
#define PetscMemcpy(d, s, n) (memcpy((d), (s), (n)), 0)
PetscErrorCode PetscGlobalMax(MPI_Comm c, const PetscReal *l, PetscReal *g);
PetscErrorCode PetscGlobalMin(MPI_Comm c, const PetscReal *l, PetscReal *g);
PetscErrorCode PetscGlobalSum(MPI_Comm c, const PetscReal *l, PetscReal *g);

/* ---- MPI (one rank) ---- */
int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Bcast(void *b, int count, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Comm_rank(MPI_Comm c, int *r);
int MPI_Comm_size(MPI_Comm c, int *s);
int MPI_Barrier(MPI_Comm c);

/* ---- Vec ---- */
PetscErrorCode VecDuplicate(Vec v, Vec *out);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecSet(Vec v, PetscScalar a);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y);
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecAYPX(Vec y, PetscScalar b, Vec x);
PetscErrorCode VecAXPBY(Vec y, PetscScalar a, PetscScalar b, Vec x);
PetscErrorCode VecAXPBYPCZ(Vec z, PetscScalar a, PetscScalar b, PetscScalar c, Vec x, Vec y);
PetscErrorCode VecScale(Vec x, PetscScalar a);
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal *r);
PetscErrorCode VecMax(Vec x, PetscInt *idx, PetscReal *r);
PetscErrorCode VecMin(Vec x, PetscInt *idx, PetscReal *r);
PetscErrorCode VecSum(Vec x, PetscScalar *r);
PetscErrorCode VecStrideSet(Vec v, PetscInt field, PetscScalar a);
PetscErrorCode VecGetSize(Vec v, PetscInt *n);
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n);
PetscErrorCode VecGetArray(Vec v, PetscScalar **a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a);
PetscErrorCode VecPointwiseMult(Vec w, Vec x, Vec y);
PetscErrorCode VecShift(Vec v, PetscScalar a);

/* ---- DM / DMDA ---- */
PetscErrorCode DMDACreate3d(MPI_Comm c, DMBoundaryType bx, DMBoundaryType by, DMBoundaryType bz,
                            DMDAStencilType st, PetscInt M, PetscInt N, PetscInt P, PetscInt m,
                            PetscInt n, PetscInt p, PetscInt dof, PetscInt s, const PetscInt *lx,
                            const PetscInt *ly, const PetscInt *lz, DM *da);
PetscErrorCode DMSetFromOptions(DM dm);
PetscErrorCode DMSetUp(DM dm);
PetscErrorCode DMDestroy(DM *dm);
PetscErrorCode DMCreateGlobalVector(DM dm, Vec *v);
PetscErrorCode DMCreateLocalVector(DM dm, Vec *v);
PetscErrorCode DMDAGetLocalInfo(DM dm, DMDALocalInfo *info);
PetscErrorCode DMDAGetInfo(DM dm, PetscInt *dim, PetscInt *M, PetscInt *N, PetscInt *P, PetscInt *m,
                           PetscInt *n, PetscInt *p, PetscInt *dof, PetscInt *s, DMBoundaryType *bx,
                           DMBoundaryType *by, DMBoundaryType *bz, DMDAStencilType *st);
PetscErrorCode DMDAGetCorners(DM dm, PetscInt *x, PetscInt *y, PetscInt *z, PetscInt *m, PetscInt *n, PetscInt *p);
PetscErrorCode DMDAGetGhostCorners(DM dm, PetscInt *x, PetscInt *y, PetscInt *z, PetscInt *m, PetscInt *n, PetscInt *p);
PetscErrorCode DMDAVecGetArray(DM dm, Vec v, void *array);
PetscErrorCode DMDAVecRestoreArray(DM dm, Vec v, void *array);
PetscErrorCode DMGlobalToLocalBegin(DM dm, Vec g, InsertMode mode, Vec l);
PetscErrorCode DMGlobalToLocalEnd(DM dm, Vec g, InsertMode mode, Vec l);
PetscErrorCode DMLocalToGlobalBegin(DM dm, Vec l, InsertMode mode, Vec g);
PetscErrorCode DMLocalToGlobalEnd(DM dm, Vec l, InsertMode mode, Vec g);
PetscErrorCode DMLocalToLocalBegin(DM dm, Vec a, InsertMode mode, Vec b);
PetscErrorCode DMLocalToLocalEnd(DM dm, Vec a, InsertMode mode, Vec b);
PetscErrorCode DMDASetUniformCoordinates(DM dm, PetscReal x0, PetscReal x1, PetscReal y0, PetscReal y1, PetscReal z0, PetscReal z1);
PetscErrorCode DMGetCoordinateDM(DM dm, DM *cdm);
PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec *c);
PetscErrorCode DMGetCoordinates(DM dm, Vec *c);

/* ---- objects and the binary viewer (checkpoint files, main.c:215-304) ---- */
typedef struct _p_PetscObject *PetscObject;
#define PETSCVIEWERVTK "vtk"
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm c, const char *name, PetscFileMode mode, PetscViewer *v);
PetscErrorCode PetscViewerDestroy(PetscViewer *v);
PetscErrorCode VecView(Vec x, PetscViewer v);
PetscErrorCode VecLoad(Vec x, PetscViewer v);
PetscErrorCode PetscViewerCreate(MPI_Comm c, PetscViewer *v);
PetscErrorCode PetscViewerSetType(PetscViewer v, const char *t);
PetscErrorCode PetscViewerFileSetMode(PetscViewer v, PetscFileMode m);
PetscErrorCode PetscViewerFileSetName(PetscViewer v, const char *n);
PetscErrorCode PetscObjectSetName(PetscObject o, const char *n);
PetscErrorCode PetscObjectSetOptionsPrefix(PetscObject o, const char *p);
PetscErrorCode PetscOptionsClearValue(void *o, const char *n);

#endif
