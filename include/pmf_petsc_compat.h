/*
 * pmf_petsc_compat.h -- the subset of the PETSc / SLEPc / MPI C interface that
 * PreMixFEM_3D.h and driver programs written against it use, implemented by
 * libpremixfem_b200.so on one GPU (no PETSc, SLEPc or MPI installation).
 *
 * Handles (DM, Vec, Mat, KSP, PC) are opaque pointers to this library's own
 * objects.  A DM is a 3-D DMDA with one process (DMDAGetCorners returns the
 * whole mesh); a Vec owns a host array (what DMDAVecGetArray / VecGetArray
 * expose) and a device mirror used by MatMult and the preconditioner; KSP
 * implements KSPCG only.  PetscInt is 32-bit and PetscScalar a real double,
 * the configuration the reference was built with (its MPI calls pass
 * PetscInt as MPI_INT and PetscScalar as MPI_DOUBLE, src/PreMixFEM_3D.c:405,1947).
 *
 * Error handling follows PETSc: every function returns a PetscErrorCode
 * (0 = success) and PetscCall() propagates a non-zero code to the caller.
 */
#ifndef PMF_PETSC_COMPAT_H
#define PMF_PETSC_COMPAT_H

#include <stdio.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int PetscErrorCode;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef double PetscLogDouble;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;

typedef int MPI_Comm;
typedef int MPI_Datatype;
#define MPI_INT ((MPI_Datatype)1)
#define MPI_DOUBLE ((MPI_Datatype)2)
#define PETSC_COMM_WORLD ((MPI_Comm)0)
#define PETSC_COMM_SELF ((MPI_Comm)1)
#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_DETERMINE PETSC_DECIDE

#define PETSC_ERR_ARG_WRONG 62
#define PETSC_ERR_ARG_WRONGSTATE 73
#define PETSC_ERR_SUP 56
#define PETSC_ERR_LIB 76
#define PETSC_ERR_USER 83
#define PETSC_ERR_MEM 55

typedef struct _p_DM* DM;
typedef struct _p_Vec* Vec;
typedef struct _p_Mat* Mat;
typedef struct _p_KSP* KSP;
typedef struct _p_PC* PC;

typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_INFINITY = 3 } NormType;
typedef enum {
  KSP_NORM_DEFAULT = -1,
  KSP_NORM_NONE = 0,
  KSP_NORM_PRECONDITIONED = 1,
  KSP_NORM_UNPRECONDITIONED = 2,
  KSP_NORM_NATURAL = 3
} KSPNormType;
typedef enum {
  KSP_CONVERGED_ITERATING = 0,
  KSP_CONVERGED_RTOL = 2,
  KSP_CONVERGED_ATOL = 3,
  KSP_DIVERGED_ITS = -3,
  KSP_DIVERGED_NANORINF = -9,
  KSP_DIVERGED_INDEFINITE_MAT = -10
} KSPConvergedReason;
typedef const char* KSPType;
typedef const char* PCType;
#define KSPCG "cg"
#define KSPPREONLY "preonly"
#define PCSHELL "shell"
#define PCNONE "none"
#define PCJACOBI "jacobi"

/* ---- error plumbing ------------------------------------------------------------------ */
PetscErrorCode PetscError_pmf(int line, const char* func, const char* file, PetscErrorCode n, const char* fmt, ...);
#define PetscFunctionBeginUser do { } while (0)
#define PetscFunctionBegin do { } while (0)
#define PetscFunctionReturn(x) return (x)
#define PetscCall(...)                                                                \
  do {                                                                                \
    PetscErrorCode ierr_pmf_ = (__VA_ARGS__);                                         \
    if (ierr_pmf_) return PetscError_pmf(__LINE__, __func__, __FILE__, ierr_pmf_, " "); \
  } while (0)
#define PetscCallMPI(...) PetscCall(__VA_ARGS__)
#define PetscCheck(cond, comm, n, ...)                                          \
  do {                                                                          \
    if (!(cond)) return PetscError_pmf(__LINE__, __func__, __FILE__, n, __VA_ARGS__); \
  } while (0)
#define PetscMax(a, b) (((a) < (b)) ? (b) : (a))
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
/* PETSc's integer power of an integer (petscmath.h), used by src/Expe_scal.c:28
   and src/Expe_frac.c:26 for the permeability 10^cr: the base converts to
   PetscInt, the result is exact while it fits in PetscInt.  A negative power
   gives 0 (the integer part of 1 / base^|power| for |base| > 1). */
static inline PetscInt PetscPowInt(PetscInt base, PetscInt power) {
  PetscInt result = 1;
  if (power < 0) return (base == 1 || base == -1) ? ((-power) % 2 ? base : 1) : 0;
  while (power) {
    if (power & 1) result *= base;
    power >>= 1;
    if (power) base *= base;
  }
  return result;
}

/* ---- initialisation, options, output, timing ---------------------------------------------- */
PetscErrorCode PetscInitialize(int* argc, char*** argv, const char* file, const char* help);
PetscErrorCode SlepcInitialize(int* argc, char*** argv, const char* file, const char* help);
PetscErrorCode PetscFinalize(void);
PetscErrorCode SlepcFinalize(void);
PetscErrorCode PetscOptionsSetValue(void* options, const char* name, const char* value);
PetscErrorCode PetscOptionsGetInt(void* options, const char* pre, const char* name, PetscInt* ivalue, PetscBool* set);
PetscErrorCode PetscOptionsGetScalar(void* options, const char* pre, const char* name, PetscScalar* dvalue,
                                     PetscBool* set);
PetscErrorCode PetscOptionsGetReal(void* options, const char* pre, const char* name, PetscReal* dvalue,
                                   PetscBool* set);
PetscErrorCode PetscOptionsHasName(void* options, const char* pre, const char* name, PetscBool* set);
PetscErrorCode PetscPrintf(MPI_Comm comm, const char* format, ...);
PetscErrorCode PetscTime(PetscLogDouble* t);
PetscErrorCode PetscTimeSubtract(PetscLogDouble* t);
PetscErrorCode PetscMalloc_pmf(size_t bytes, void** ptr);
PetscErrorCode PetscFree_pmf(void* ptr);
#define PetscMalloc1(n, p) PetscMalloc_pmf((size_t)(n) * sizeof(**(p)), (void**)(p))
#define PetscFree(p) (PetscFree_pmf((void*)(p)), (p) = NULL, 0)
#define PetscMemzero(p, n) (memset((p), 0, (n)), 0)
#define PetscArraycpy(dst, src, n) (memcpy((dst), (src), (size_t)(n) * sizeof(*(dst))), 0)

/* ---- DMDA (3-D, star stencil, one process) ---------------------------------------------- */
typedef enum { DM_BOUNDARY_NONE = 0 } DMBoundaryType;
typedef enum { DMDA_STENCIL_STAR = 0, DMDA_STENCIL_BOX = 1 } DMDAStencilType;
PetscErrorCode DMDACreate3d(MPI_Comm comm, DMBoundaryType bx, DMBoundaryType by, DMBoundaryType bz,
                            DMDAStencilType st, PetscInt M, PetscInt N, PetscInt P, PetscInt m, PetscInt n,
                            PetscInt p, PetscInt dof, PetscInt s, const PetscInt lx[], const PetscInt ly[],
                            const PetscInt lz[], DM* da);
PetscErrorCode DMSetUp(DM dm);
PetscErrorCode DMDestroy(DM* dm);
PetscErrorCode DMDAGetCorners(DM dm, PetscInt* x, PetscInt* y, PetscInt* z, PetscInt* m, PetscInt* n, PetscInt* p);
PetscErrorCode DMDAGetInfo(DM dm, PetscInt* dim, PetscInt* M, PetscInt* N, PetscInt* P, PetscInt* m, PetscInt* n,
                           PetscInt* p, PetscInt* dof, PetscInt* s, DMBoundaryType* bx, DMBoundaryType* by,
                           DMBoundaryType* bz, DMDAStencilType* st);
PetscErrorCode DMCreateGlobalVector(DM dm, Vec* v);
PetscErrorCode DMCreateLocalVector(DM dm, Vec* v);
/* array is PetscScalar*** indexed [k][j][i] (z, y, x) */
PetscErrorCode DMDAVecGetArray(DM dm, Vec v, void* array);
PetscErrorCode DMDAVecRestoreArray(DM dm, Vec v, void* array);
PetscErrorCode DMDAVecGetArrayRead(DM dm, Vec v, void* array);
PetscErrorCode DMDAVecRestoreArrayRead(DM dm, Vec v, void* array);

/* ---- Vec --------------------------------------------------------------------------------- */
PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec* v);
PetscErrorCode VecDuplicate(Vec v, Vec* newv);
PetscErrorCode VecDestroy(Vec* v);
PetscErrorCode VecGetSize(Vec v, PetscInt* n);
PetscErrorCode VecSet(Vec v, PetscScalar alpha);
PetscErrorCode VecZeroEntries(Vec v);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecAXPY(Vec y, PetscScalar alpha, Vec x);
PetscErrorCode VecAYPX(Vec y, PetscScalar beta, Vec x);
PetscErrorCode VecScale(Vec x, PetscScalar alpha);
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar* val);
PetscErrorCode VecNorm(Vec x, NormType type, PetscReal* val);
PetscErrorCode VecNormalize(Vec x, PetscReal* val);
PetscErrorCode VecGetArray(Vec x, PetscScalar** a);
PetscErrorCode VecRestoreArray(Vec x, PetscScalar** a);
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar** a);
PetscErrorCode VecRestoreArrayRead(Vec x, const PetscScalar** a);

/* ---- Mat (the operator of PC_create_A, matrix-free on the GPU) ---------------------------- */
PetscErrorCode MatMult(Mat A, Vec x, Vec y);
PetscErrorCode MatDestroy(Mat* A);
PetscErrorCode MatGetSize(Mat A, PetscInt* m, PetscInt* n);

/* ---- KSP / PC ---------------------------------------------------------------------------------- */
PetscErrorCode KSPCreate(MPI_Comm comm, KSP* ksp);
PetscErrorCode KSPSetOperators(KSP ksp, Mat Amat, Mat Pmat);
PetscErrorCode KSPSetType(KSP ksp, KSPType type);
PetscErrorCode KSPGetPC(KSP ksp, PC* pc);
PetscErrorCode KSPSetNormType(KSP ksp, KSPNormType normtype);
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal abstol, PetscReal dtol, PetscInt maxits);
/* reads -ksp_type, -pc_type, -ksp_rtol, -ksp_atol, -ksp_divtol, -ksp_max_it,
 * -ksp_norm_type, -ksp_monitor, -ksp_converged_reason and
 * -ksp_constant_null_space (constant null space of the operator) */
PetscErrorCode KSPSetFromOptions(KSP ksp);
PetscErrorCode KSPSetUp(KSP ksp);
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt* its);
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal* rnorm);
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason* reason);
PetscErrorCode KSPConvergedReasonView(KSP ksp, void* viewer);
PetscErrorCode KSPDestroy(KSP* ksp);
PetscErrorCode PCSetType(PC pc, PCType type);
PetscErrorCode PCShellSetContext(PC pc, void* ctx);
PetscErrorCode PCShellGetContext(PC pc, void* ctx);
PetscErrorCode PCShellSetSetUp(PC pc, PetscErrorCode (*setup)(PC));
PetscErrorCode PCShellSetApply(PC pc, PetscErrorCode (*apply)(PC, Vec, Vec));
PetscErrorCode PCShellSetName(PC pc, const char* name);
PetscErrorCode PCGetOperators(PC pc, Mat* Amat, Mat* Pmat);

#ifdef __cplusplus
}
#endif

#endif
