// The reference's public C interface (PreMixFEM_3D.h) and the PETSc subset
// its drivers call (pmf_petsc_compat.h), implemented on one GPU.
//
// A DM made by PC_init owns a pmf::Solver; every other object is a thin host
// handle.  Vec data live in pinned host memory (what DMDAVecGetArray and
// VecGetArray expose); MatMult, PC_setup, PC_apply_vec and KSPSolve move them
// to the device per call.  KSPSolve of a KSPCG whose shell apply is
// PC_apply_vec, with the unpreconditioned norm the reference selects
// (src/Expe_scal.c, KSPSetNormType), runs the whole CG on the device
// (Solver::solve); any other PC or norm type runs PETSc's CG recurrence on the
// host over the same MatMult / PC callbacks.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "PreMixFEM_3D.h"
#include "solver.h"

// ------------------------------------------------------------------------------------------
// objects
struct _p_DM {
  PetscInt M = 0, N = 0, P = 0;
  pmf::Solver* solver = nullptr;  // set by PC_init
};

struct _p_Vec {
  PetscInt n = 0;
  double* a = nullptr;
  bool pinned = false;
  PetscInt M = 0, N = 0, P = 0;  // DMDA shape (0 for VecCreateSeq)
  std::vector<double*> rows;
  std::vector<double**> planes;
};

struct _p_Mat {
  DM dm = nullptr;
};

struct _p_PC {
  std::string type = PCNONE;
  void* ctx = nullptr;
  PetscErrorCode (*setup)(PC) = nullptr;
  PetscErrorCode (*apply)(PC, Vec, Vec) = nullptr;
  std::string name;
  KSP ksp = nullptr;
  bool is_setup = false;
  std::vector<double> jacobi;  // inverse diagonal for PCJACOBI
};

struct _p_KSP {
  Mat A = nullptr, Pm = nullptr;
  _p_PC pc;
  std::string type = KSPCG;
  KSPNormType norm = KSP_NORM_DEFAULT;
  double rtol = 1e-5, atol = 1e-50, dtol = 1e5;
  int max_it = 10000;
  bool is_setup = false, monitor = false, view_reason = false;
  bool null_space = false;  // -ksp_constant_null_space: constant null space on the operator
  int its = 0;
  double rnorm = 0.0;
  KSPConvergedReason reason = KSP_CONVERGED_ITERATING;
};

// ------------------------------------------------------------------------------------------
// options database and error plumbing
static pmf::OptionDB g_db;

static const char* strip_dash(const char* name) { return (name && name[0] == '-') ? name + 1 : name; }

static bool looks_like_value(const char* t) {
  if (!t || !t[0]) return false;
  if (t[0] != '-') return true;
  return (t[1] >= '0' && t[1] <= '9') || t[1] == '.';  // a negative number
}

static void parse_args(int argc, char** argv) {
  for (int i = 1; i < argc; ++i) {
    const char* t = argv[i];
    if (!t || t[0] != '-') continue;
    std::string key = strip_dash(t);
    std::string val;
    if (i + 1 < argc && looks_like_value(argv[i + 1])) val = argv[++i];
    g_db.kv[key] = val;
  }
}

extern "C" {

PetscErrorCode PetscError_pmf(int line, const char* func, const char* file, PetscErrorCode n, const char* fmt, ...) {
  char msg[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof(msg), fmt ? fmt : "", ap);
  va_end(ap);
  fprintf(stderr, "[premixfem_b200] error %d in %s() at %s:%d: %s\n", n, func ? func : "?", file ? file : "?", line,
          msg);
  return n;
}

#define SHIM_ERR(n, ...) PetscError_pmf(__LINE__, __func__, __FILE__, n, __VA_ARGS__)

PetscErrorCode PetscInitialize(int* argc, char*** argv, const char* file, const char* help) {
  (void)file;
  (void)help;
  if (const char* env = getenv("PETSC_OPTIONS")) g_db.parse(env);
  if (argc && argv) parse_args(*argc, *argv);
  return 0;
}
PetscErrorCode SlepcInitialize(int* argc, char*** argv, const char* file, const char* help) {
  return PetscInitialize(argc, argv, file, help);
}
PetscErrorCode PetscFinalize(void) {
  g_db.kv.clear();
  return 0;
}
PetscErrorCode SlepcFinalize(void) { return PetscFinalize(); }

PetscErrorCode PetscOptionsSetValue(void* options, const char* name, const char* value) {
  (void)options;
  if (!name) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null option name");
  g_db.kv[strip_dash(name)] = value ? value : "";
  return 0;
}

static const std::string* find_opt(const char* pre, const char* name) {
  std::string key = pre ? std::string(strip_dash(pre)) + strip_dash(name) : std::string(strip_dash(name));
  auto it = g_db.kv.find(key);
  return it == g_db.kv.end() ? nullptr : &it->second;
}

PetscErrorCode PetscOptionsGetInt(void* options, const char* pre, const char* name, PetscInt* ivalue, PetscBool* set) {
  (void)options;
  const std::string* v = find_opt(pre, name);
  if (set) *set = PETSC_FALSE;
  if (!v) return 0;
  if (v->empty()) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "option %s needs an integer value", name);
  char* end = nullptr;
  long x = strtol(v->c_str(), &end, 10);
  if (!end || *end) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "option %s: '%s' is not an integer", name, v->c_str());
  if (ivalue) *ivalue = (PetscInt)x;
  if (set) *set = PETSC_TRUE;
  return 0;
}

PetscErrorCode PetscOptionsGetReal(void* options, const char* pre, const char* name, PetscReal* dvalue,
                                   PetscBool* set) {
  (void)options;
  const std::string* v = find_opt(pre, name);
  if (set) *set = PETSC_FALSE;
  if (!v) return 0;
  if (v->empty()) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "option %s needs a real value", name);
  char* end = nullptr;
  double x = strtod(v->c_str(), &end);
  if (!end || *end) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "option %s: '%s' is not a number", name, v->c_str());
  if (dvalue) *dvalue = x;
  if (set) *set = PETSC_TRUE;
  return 0;
}

PetscErrorCode PetscOptionsGetScalar(void* options, const char* pre, const char* name, PetscScalar* dvalue,
                                     PetscBool* set) {
  return PetscOptionsGetReal(options, pre, name, dvalue, set);
}

PetscErrorCode PetscOptionsHasName(void* options, const char* pre, const char* name, PetscBool* set) {
  (void)options;
  const std::string* v = find_opt(pre, name);
  bool on = v != nullptr;
  if (v && (*v == "0" || *v == "false" || *v == "no")) on = false;
  if (set) *set = on ? PETSC_TRUE : PETSC_FALSE;
  return 0;
}

PetscErrorCode PetscPrintf(MPI_Comm comm, const char* format, ...) {
  (void)comm;
  va_list ap;
  va_start(ap, format);
  vprintf(format, ap);
  va_end(ap);
  fflush(stdout);
  return 0;
}

static double wall_seconds() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}
PetscErrorCode PetscTime(PetscLogDouble* t) {
  *t = wall_seconds();
  return 0;
}
PetscErrorCode PetscTimeSubtract(PetscLogDouble* t) {
  *t -= wall_seconds();
  return 0;
}

PetscErrorCode PetscMalloc_pmf(size_t bytes, void** ptr) {
  *ptr = bytes ? malloc(bytes) : nullptr;
  if (bytes && !*ptr) return SHIM_ERR(PETSC_ERR_MEM, "out of host memory (%zu bytes)", bytes);
  return 0;
}
PetscErrorCode PetscFree_pmf(void* ptr) {
  free(ptr);
  return 0;
}

// ------------------------------------------------------------------------------------------
// DMDA
PetscErrorCode DMDACreate3d(MPI_Comm comm, DMBoundaryType bx, DMBoundaryType by, DMBoundaryType bz,
                            DMDAStencilType st, PetscInt M, PetscInt N, PetscInt P, PetscInt m, PetscInt n,
                            PetscInt p, PetscInt dof, PetscInt s, const PetscInt lx[], const PetscInt ly[],
                            const PetscInt lz[], DM* da) {
  (void)comm;
  (void)st;
  (void)s;
  (void)lx;
  (void)ly;
  (void)lz;
  if (!da) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null DM pointer");
  if (bx != DM_BOUNDARY_NONE || by != DM_BOUNDARY_NONE || bz != DM_BOUNDARY_NONE)
    return SHIM_ERR(PETSC_ERR_SUP, "only DM_BOUNDARY_NONE is supported");
  if (dof != 1) return SHIM_ERR(PETSC_ERR_SUP, "only dof=1 is supported");
  if ((m > 1) || (n > 1) || (p > 1))
    return SHIM_ERR(PETSC_ERR_SUP, "one process owns the whole DMDA (use -pmf_vranks for the rank grid)");
  if (M < 1 || N < 1 || P < 1) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "bad DMDA size %d x %d x %d", M, N, P);
  DM d = new _p_DM;
  d->M = M;
  d->N = N;
  d->P = P;
  *da = d;
  return 0;
}
PetscErrorCode DMSetUp(DM dm) {
  return dm ? 0 : SHIM_ERR(PETSC_ERR_ARG_WRONG, "null DM");
}
PetscErrorCode DMDestroy(DM* dm) {
  if (!dm || !*dm) return 0;
  delete (*dm)->solver;
  delete *dm;
  *dm = nullptr;
  return 0;
}
PetscErrorCode DMDAGetCorners(DM dm, PetscInt* x, PetscInt* y, PetscInt* z, PetscInt* m, PetscInt* n, PetscInt* p) {
  if (!dm) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null DM");
  if (x) *x = 0;
  if (y) *y = 0;
  if (z) *z = 0;
  if (m) *m = dm->M;
  if (n) *n = dm->N;
  if (p) *p = dm->P;
  return 0;
}
PetscErrorCode DMDAGetInfo(DM dm, PetscInt* dim, PetscInt* M, PetscInt* N, PetscInt* P, PetscInt* m, PetscInt* n,
                           PetscInt* p, PetscInt* dof, PetscInt* s, DMBoundaryType* bx, DMBoundaryType* by,
                           DMBoundaryType* bz, DMDAStencilType* st) {
  if (!dm) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null DM");
  if (dim) *dim = 3;
  if (M) *M = dm->M;
  if (N) *N = dm->N;
  if (P) *P = dm->P;
  if (m) *m = 1;
  if (n) *n = 1;
  if (p) *p = 1;
  if (dof) *dof = 1;
  if (s) *s = 1;
  if (bx) *bx = DM_BOUNDARY_NONE;
  if (by) *by = DM_BOUNDARY_NONE;
  if (bz) *bz = DM_BOUNDARY_NONE;
  if (st) *st = DMDA_STENCIL_STAR;
  return 0;
}

static PetscErrorCode vec_alloc(PetscInt n, Vec* v) {
  if (!v) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null Vec pointer");
  if (n < 0) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "negative Vec size");
  Vec x = new _p_Vec;
  x->n = n;
  const size_t bytes = (size_t)(n > 0 ? n : 1) * sizeof(double);
  void* p = nullptr;
  // pinned memory makes the per-call host<->device copies run at full PCIe/C2C speed
  if (cudaMallocHost(&p, bytes) == cudaSuccess) {
    x->pinned = true;
  } else {
    cudaGetLastError();
    p = malloc(bytes);
    if (!p) {
      delete x;
      return SHIM_ERR(PETSC_ERR_MEM, "out of host memory for a Vec of %d entries", n);
    }
  }
  x->a = (double*)p;
  memset(x->a, 0, bytes);
  *v = x;
  return 0;
}

PetscErrorCode DMCreateGlobalVector(DM dm, Vec* v) {
  if (!dm) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null DM");
  PetscCall(vec_alloc(dm->M * dm->N * dm->P, v));
  (*v)->M = dm->M;
  (*v)->N = dm->N;
  (*v)->P = dm->P;
  return 0;
}
// one process and no periodic boundary: the local vector has no ghost points
PetscErrorCode DMCreateLocalVector(DM dm, Vec* v) { return DMCreateGlobalVector(dm, v); }

PetscErrorCode DMDAVecGetArray(DM dm, Vec v, void* array) {
  if (!dm || !v || !array) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  if (v->n != dm->M * dm->N * dm->P) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "Vec does not match the DMDA");
  if (v->planes.empty()) {
    v->rows.resize((size_t)dm->N * dm->P);
    v->planes.resize(dm->P);
    for (PetscInt k = 0; k < dm->P; ++k) {
      for (PetscInt j = 0; j < dm->N; ++j) v->rows[(size_t)k * dm->N + j] = v->a + ((size_t)k * dm->N + j) * dm->M;
      v->planes[k] = &v->rows[(size_t)k * dm->N];
    }
  }
  *(double****)array = v->planes.data();
  return 0;
}
PetscErrorCode DMDAVecRestoreArray(DM dm, Vec v, void* array) {
  (void)dm;
  (void)v;
  if (array) *(double****)array = nullptr;
  return 0;
}
PetscErrorCode DMDAVecGetArrayRead(DM dm, Vec v, void* array) { return DMDAVecGetArray(dm, v, array); }
PetscErrorCode DMDAVecRestoreArrayRead(DM dm, Vec v, void* array) { return DMDAVecRestoreArray(dm, v, array); }

// ------------------------------------------------------------------------------------------
// Vec
PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec* v) {
  (void)comm;
  return vec_alloc(n, v);
}
PetscErrorCode VecDuplicate(Vec v, Vec* newv) {
  if (!v) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null Vec");
  PetscCall(vec_alloc(v->n, newv));
  (*newv)->M = v->M;
  (*newv)->N = v->N;
  (*newv)->P = v->P;
  return 0;
}
PetscErrorCode VecDestroy(Vec* v) {
  if (!v || !*v) return 0;
  if ((*v)->pinned)
    cudaFreeHost((*v)->a);
  else
    free((*v)->a);
  delete *v;
  *v = nullptr;
  return 0;
}
PetscErrorCode VecGetSize(Vec v, PetscInt* n) {
  if (!v) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null Vec");
  *n = v->n;
  return 0;
}
PetscErrorCode VecSet(Vec v, PetscScalar alpha) {
  if (!v) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null Vec");
  for (PetscInt i = 0; i < v->n; ++i) v->a[i] = alpha;
  return 0;
}
PetscErrorCode VecZeroEntries(Vec v) { return VecSet(v, 0.0); }
static PetscErrorCode same_size(Vec x, Vec y) {
  if (!x || !y) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null Vec");
  if (x->n != y->n) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "Vec sizes differ (%d vs %d)", x->n, y->n);
  return 0;
}
PetscErrorCode VecCopy(Vec x, Vec y) {
  PetscCall(same_size(x, y));
  if (x != y) memcpy(y->a, x->a, sizeof(double) * x->n);
  return 0;
}
PetscErrorCode VecAXPY(Vec y, PetscScalar alpha, Vec x) {
  PetscCall(same_size(x, y));
  for (PetscInt i = 0; i < y->n; ++i) y->a[i] += alpha * x->a[i];
  return 0;
}
PetscErrorCode VecAYPX(Vec y, PetscScalar beta, Vec x) {
  PetscCall(same_size(x, y));
  for (PetscInt i = 0; i < y->n; ++i) y->a[i] = x->a[i] + beta * y->a[i];
  return 0;
}
PetscErrorCode VecScale(Vec x, PetscScalar alpha) {
  if (!x) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null Vec");
  for (PetscInt i = 0; i < x->n; ++i) x->a[i] *= alpha;
  return 0;
}
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar* val) {
  PetscCall(same_size(x, y));
  double s = 0.0;
  for (PetscInt i = 0; i < x->n; ++i) s += x->a[i] * y->a[i];
  *val = s;
  return 0;
}
PetscErrorCode VecNorm(Vec x, NormType type, PetscReal* val) {
  if (!x) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null Vec");
  double s = 0.0;
  if (type == NORM_1) {
    for (PetscInt i = 0; i < x->n; ++i) s += fabs(x->a[i]);
  } else if (type == NORM_INFINITY) {
    for (PetscInt i = 0; i < x->n; ++i) s = fmax(s, fabs(x->a[i]));
  } else if (type == NORM_2) {
    for (PetscInt i = 0; i < x->n; ++i) s += x->a[i] * x->a[i];
    s = sqrt(s);
  } else {
    return SHIM_ERR(PETSC_ERR_SUP, "unsupported NormType %d", (int)type);
  }
  *val = s;
  return 0;
}
PetscErrorCode VecNormalize(Vec x, PetscReal* val) {
  double nrm = 0.0;
  PetscCall(VecNorm(x, NORM_2, &nrm));
  if (nrm != 0.0) PetscCall(VecScale(x, 1.0 / nrm));
  if (val) *val = nrm;
  return 0;
}
PetscErrorCode VecGetArray(Vec x, PetscScalar** a) {
  if (!x || !a) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  *a = x->a;
  return 0;
}
PetscErrorCode VecRestoreArray(Vec x, PetscScalar** a) {
  (void)x;
  if (a) *a = nullptr;
  return 0;
}
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar** a) {
  if (!x || !a) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  *a = x->a;
  return 0;
}
PetscErrorCode VecRestoreArrayRead(Vec x, const PetscScalar** a) {
  (void)x;
  if (a) *a = nullptr;
  return 0;
}

// ------------------------------------------------------------------------------------------
// Mat: the 7-point operator held by the DM's solver
static PetscErrorCode solver_call(pmf::Solver* s, int code) {
  if (code) return SHIM_ERR(code, "%s", s ? s->err.c_str() : "no solver");
  return 0;
}

PetscErrorCode MatMult(Mat A, Vec x, Vec y) {
  if (!A || !A->dm || !A->dm->solver) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "Mat was not made by PC_create_A");
  PetscCall(same_size(x, y));
  if (x->n != A->dm->M * A->dm->N * A->dm->P) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "Vec does not match the Mat");
  if (x == y) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "x and y must be different vectors");
  return solver_call(A->dm->solver, A->dm->solver->apply_A(x->a, y->a, false));
}
PetscErrorCode MatDestroy(Mat* A) {
  if (!A || !*A) return 0;
  delete *A;
  *A = nullptr;
  return 0;
}
PetscErrorCode MatGetSize(Mat A, PetscInt* m, PetscInt* n) {
  if (!A || !A->dm) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null Mat");
  const PetscInt sz = A->dm->M * A->dm->N * A->dm->P;
  if (m) *m = sz;
  if (n) *n = sz;
  return 0;
}

// ------------------------------------------------------------------------------------------
// PC
PetscErrorCode PCSetType(PC pc, PCType type) {
  if (!pc || !type) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  std::string t = type;
  if (t != PCSHELL && t != PCNONE && t != PCJACOBI)
    return SHIM_ERR(PETSC_ERR_SUP, "PC type '%s' is not provided (shell, none, jacobi)", type);
  pc->type = t;
  pc->is_setup = false;
  return 0;
}
PetscErrorCode PCShellSetContext(PC pc, void* ctx) {
  if (!pc) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null PC");
  pc->ctx = ctx;
  return 0;
}
PetscErrorCode PCShellGetContext(PC pc, void* ctx) {
  if (!pc || !ctx) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  *(void**)ctx = pc->ctx;
  return 0;
}
PetscErrorCode PCShellSetSetUp(PC pc, PetscErrorCode (*setup)(PC)) {
  if (!pc) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null PC");
  pc->setup = setup;
  return 0;
}
PetscErrorCode PCShellSetApply(PC pc, PetscErrorCode (*apply)(PC, Vec, Vec)) {
  if (!pc) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null PC");
  pc->apply = apply;
  return 0;
}
PetscErrorCode PCShellSetName(PC pc, const char* name) {
  if (!pc) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null PC");
  pc->name = name ? name : "";
  return 0;
}
PetscErrorCode PCGetOperators(PC pc, Mat* Amat, Mat* Pmat) {
  if (!pc || !pc->ksp) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "PC has no KSP");
  if (Amat) *Amat = pc->ksp->A;
  if (Pmat) *Pmat = pc->ksp->Pm;
  return 0;
}

static PetscErrorCode pc_setup(PC pc) {
  if (pc->is_setup) return 0;
  if (pc->type == PCSHELL) {
    if (pc->setup) PetscCall(pc->setup(pc));
  } else if (pc->type == PCJACOBI) {
    Mat A = pc->ksp->Pm ? pc->ksp->Pm : pc->ksp->A;
    pmf::Solver* s = A->dm->solver;
    const size_t n = (size_t)s->g.ncell;
    pc->jacobi.resize(n);
    if (cudaMemcpy(pc->jacobi.data(), s->diag, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
      return SHIM_ERR(PETSC_ERR_LIB, "reading the operator diagonal failed");
    for (auto& d : pc->jacobi) d = d != 0.0 ? 1.0 / d : 1.0;
  }
  pc->is_setup = true;
  return 0;
}

static PetscErrorCode pc_apply(PC pc, Vec x, Vec y) {
  if (pc->type == PCSHELL) {
    if (!pc->apply) return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "PCSHELL without an apply function");
    return pc->apply(pc, x, y);
  }
  if (pc->type == PCJACOBI) {
    for (PetscInt i = 0; i < x->n; ++i) y->a[i] = pc->jacobi[i] * x->a[i];
    return 0;
  }
  return VecCopy(x, y);
}

// ------------------------------------------------------------------------------------------
// KSP (CG only)
PetscErrorCode KSPCreate(MPI_Comm comm, KSP* ksp) {
  (void)comm;
  if (!ksp) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null KSP pointer");
  KSP k = new _p_KSP;
  k->pc.ksp = k;
  *ksp = k;
  return 0;
}
PetscErrorCode KSPSetOperators(KSP ksp, Mat Amat, Mat Pmat) {
  if (!ksp || !Amat) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  ksp->A = Amat;
  ksp->Pm = Pmat ? Pmat : Amat;
  ksp->is_setup = false;
  ksp->pc.is_setup = false;
  return 0;
}
PetscErrorCode KSPSetType(KSP ksp, KSPType type) {
  if (!ksp || !type) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  if (strcmp(type, KSPCG) != 0) return SHIM_ERR(PETSC_ERR_SUP, "KSP type '%s' is not provided (cg only)", type);
  ksp->type = type;
  return 0;
}
PetscErrorCode KSPGetPC(KSP ksp, PC* pc) {
  if (!ksp || !pc) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  *pc = &ksp->pc;
  return 0;
}
PetscErrorCode KSPSetNormType(KSP ksp, KSPNormType normtype) {
  if (!ksp) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null KSP");
  ksp->norm = normtype;
  return 0;
}
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal abstol, PetscReal dtol, PetscInt maxits) {
  if (!ksp) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null KSP");
  if (rtol != PETSC_DEFAULT) ksp->rtol = rtol;
  if (abstol != PETSC_DEFAULT) ksp->atol = abstol;
  if (dtol != PETSC_DEFAULT) ksp->dtol = dtol;
  if (maxits != PETSC_DEFAULT) ksp->max_it = maxits;
  return 0;
}
PetscErrorCode KSPSetFromOptions(KSP ksp) {
  if (!ksp) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null KSP");
  if (const std::string* t = find_opt(nullptr, "ksp_type")) PetscCall(KSPSetType(ksp, t->c_str()));
  if (const std::string* t = find_opt(nullptr, "pc_type")) PetscCall(PCSetType(&ksp->pc, t->c_str()));
  PetscCall(PetscOptionsGetReal(nullptr, nullptr, "-ksp_rtol", &ksp->rtol, nullptr));
  PetscCall(PetscOptionsGetReal(nullptr, nullptr, "-ksp_atol", &ksp->atol, nullptr));
  PetscCall(PetscOptionsGetReal(nullptr, nullptr, "-ksp_divtol", &ksp->dtol, nullptr));
  PetscCall(PetscOptionsGetInt(nullptr, nullptr, "-ksp_max_it", &ksp->max_it, nullptr));
  if (const std::string* t = find_opt(nullptr, "ksp_norm_type")) {
    if (*t == "unpreconditioned")
      ksp->norm = KSP_NORM_UNPRECONDITIONED;
    else if (*t == "preconditioned")
      ksp->norm = KSP_NORM_PRECONDITIONED;
    else if (*t == "natural")
      ksp->norm = KSP_NORM_NATURAL;
    else if (*t == "none")
      ksp->norm = KSP_NORM_NONE;
    else
      return SHIM_ERR(PETSC_ERR_ARG_WRONG, "unknown -ksp_norm_type %s", t->c_str());
  }
  if (const std::string* t = find_opt(nullptr, "ksp_constant_null_space")) {
    // PetscOptionsBool: the bare flag or true/yes/on/1 sets it, false/no/off/0 clears it
    if (t->empty() || *t == "1" || *t == "true" || *t == "yes" || *t == "on")
      ksp->null_space = true;
    else if (*t == "0" || *t == "false" || *t == "no" || *t == "off")
      ksp->null_space = false;
    else
      return SHIM_ERR(PETSC_ERR_ARG_WRONG, "unknown -ksp_constant_null_space %s", t->c_str());
  }
  PetscBool b = PETSC_FALSE;
  PetscCall(PetscOptionsHasName(nullptr, nullptr, "-ksp_monitor", &b));
  ksp->monitor = b;
  PetscCall(PetscOptionsHasName(nullptr, nullptr, "-ksp_converged_reason", &b));
  ksp->view_reason = b;
  return 0;
}
PetscErrorCode KSPSetUp(KSP ksp) {
  if (!ksp || !ksp->A) return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "KSPSetOperators must come first");
  if (ksp->is_setup) return 0;
  PetscCall(pc_setup(&ksp->pc));
  ksp->is_setup = true;
  return 0;
}

static const char* reason_name(KSPConvergedReason r) {
  switch (r) {
    case KSP_CONVERGED_RTOL: return "CONVERGED_RTOL";
    case KSP_CONVERGED_ATOL: return "CONVERGED_ATOL";
    case KSP_DIVERGED_ITS: return "DIVERGED_ITS";
    case KSP_DIVERGED_NANORINF: return "DIVERGED_NANORINF";
    case KSP_DIVERGED_INDEFINITE_MAT: return "DIVERGED_INDEFINITE_MAT";
    default: return "CONVERGED_ITERATING";
  }
}

// PETSc's KSPSolve_CG recurrence (zero initial guess) over the host callbacks:
// with the unpreconditioned norm the residual is tested before the next
// preconditioner application; with the preconditioned / natural norm after it.
static PetscErrorCode cg_host(KSP ksp, Vec b, Vec x) {
  const PetscInt n = b->n;
  Vec r, z, p, w;
  PetscCall(VecDuplicate(b, &r));
  PetscCall(VecDuplicate(b, &z));
  PetscCall(VecDuplicate(b, &p));
  PetscCall(VecDuplicate(b, &w));
  PetscErrorCode ierr = 0;
  const bool unprec = ksp->norm == KSP_NORM_UNPRECONDITIONED;
  const bool natural = ksp->norm == KSP_NORM_NATURAL;
  auto norm2 = [&](Vec v) {
    double t = 0.0;
    for (PetscInt i = 0; i < n; ++i) t += v->a[i] * v->a[i];
    return sqrt(t);
  };
  // KSP_PCApply: the preconditioner, then MatNullSpaceRemove of the constant
  // null space (z <- z - (sum z / n) 1) when the operator carries one
  auto precondition = [&](Vec rr, Vec zz) -> PetscErrorCode {
    PetscErrorCode e = pc_apply(&ksp->pc, rr, zz);
    if (e || !ksp->null_space || n == 0) return e;
    double sum = 0.0;
    for (PetscInt i = 0; i < n; ++i) sum += zz->a[i];
    const double shift = sum / (-(double)n);
    for (PetscInt i = 0; i < n; ++i) zz->a[i] += shift;
    return 0;
  };
  double beta = 0.0, betaold = 0.0, dp = 0.0, ttol = 0.0, dpi = 0.0, dpiold = 0.0;
  // residual test; returns true when the iteration stops
  auto test = [&](int it) {
    if (ksp->monitor) printf("  %d KSP Residual norm %.12e\n", it, dp);
    if (!std::isfinite(dp)) {
      ksp->reason = KSP_DIVERGED_NANORINF;
      return true;
    }
    if (dp <= ttol) {
      ksp->reason = dp <= ksp->atol ? KSP_CONVERGED_ATOL : KSP_CONVERGED_RTOL;
      return true;
    }
    return false;
  };
  ksp->its = 0;
  ksp->reason = KSP_CONVERGED_ITERATING;
  VecZeroEntries(x);
  VecCopy(b, r);
  do {
    if (unprec) {
      dp = norm2(r);
      ttol = fmax(ksp->rtol * dp, ksp->atol);
      if (test(0)) break;
      if ((ierr = precondition(r, z))) break;
      VecDot(z, r, &beta);
    } else {
      if ((ierr = precondition(r, z))) break;
      VecDot(z, r, &beta);
      dp = natural ? sqrt(fabs(beta)) : norm2(z);
      ttol = fmax(ksp->rtol * dp, ksp->atol);
      if (test(0)) break;
    }
    for (int i = 0; i < ksp->max_it; ++i) {
      ksp->its = i + 1;
      if (beta == 0.0) {
        ksp->reason = KSP_CONVERGED_ATOL;
        break;
      }
      if (i == 0)
        VecCopy(z, p);
      else
        VecAYPX(p, beta / betaold, z);
      if ((ierr = MatMult(ksp->A, p, w))) break;
      dpiold = dpi;
      VecDot(p, w, &dpi);
      betaold = beta;
      if (dpi == 0.0 || (i > 0 && dpi * dpiold < 0.0)) {
        ksp->reason = KSP_DIVERGED_INDEFINITE_MAT;
        break;
      }
      const double alpha = beta / dpi;
      VecAXPY(x, alpha, p);
      VecAXPY(r, -alpha, w);
      if (unprec) {
        dp = norm2(r);
        if (test(i + 1)) break;
        if ((ierr = precondition(r, z))) break;
        VecDot(z, r, &beta);
      } else {
        if ((ierr = precondition(r, z))) break;
        VecDot(z, r, &beta);
        dp = natural ? sqrt(fabs(beta)) : norm2(z);
        if (test(i + 1)) break;
      }
    }
    if (!ierr && ksp->reason == KSP_CONVERGED_ITERATING) ksp->reason = KSP_DIVERGED_ITS;
  } while (0);
  ksp->rnorm = dp;
  VecDestroy(&r);
  VecDestroy(&z);
  VecDestroy(&p);
  VecDestroy(&w);
  return ierr;
}

PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x) {
  if (!ksp || !b || !x) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  PetscCall(same_size(b, x));
  PetscCall(KSPSetUp(ksp));
  const bool unprec = ksp->norm == KSP_NORM_UNPRECONDITIONED;
  PCCtx* ctx = (PCCtx*)ksp->pc.ctx;
  const bool ours = ksp->pc.type == PCSHELL && ksp->pc.apply == PC_apply_vec && ctx && ctx->dm &&
                    ctx->dm->solver && ksp->A->dm && ctx->dm->solver == ksp->A->dm->solver;
  if (ours && unprec) {
    pmf::Solver* s = ctx->dm->solver;
    s->opt.rtol = ksp->rtol;
    s->opt.atol = ksp->atol;
    s->opt.max_it = ksp->max_it;
    s->opt.null_space = ksp->null_space;
    int its = 0, code = 0;
    double rnorm = 0.0;
    const double av0 = s->t_stages[pmf::ST_AV];
    PetscCall(solver_call(s, s->solve(b->a, x->a, false, &its, &rnorm, &code)));
    // the device solve fuses the V-cycles with the CG vector updates; its
    // device time is booked as preconditioner application time
    ctx->t_stages[STAGE_AV] += s->last_solve_ms * 1e-3 + (s->t_stages[pmf::ST_AV] - av0);
    ksp->its = its;
    ksp->rnorm = rnorm;
    // pmf::Solver::solve stop codes -> KSPConvergedReason, as cg_host sets them
    if (code == 1)
      ksp->reason = rnorm <= ksp->atol ? KSP_CONVERGED_ATOL : KSP_CONVERGED_RTOL;
    else if (code == 5)
      ksp->reason = KSP_CONVERGED_ATOL;  // z.r = 0
    else if (code == 3)
      ksp->reason = KSP_DIVERGED_INDEFINITE_MAT;
    else if (code == 4)
      ksp->reason = KSP_DIVERGED_NANORINF;
    else
      ksp->reason = KSP_DIVERGED_ITS;  // 2, or a loop stopped by the host guard
  } else {
    PetscCall(cg_host(ksp, b, x));
  }
  if (ksp->view_reason) PetscCall(KSPConvergedReasonView(ksp, nullptr));
  return 0;
}
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt* its) {
  if (!ksp || !its) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  *its = ksp->its;
  return 0;
}
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal* rnorm) {
  if (!ksp || !rnorm) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  *rnorm = ksp->rnorm;
  return 0;
}
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason* reason) {
  if (!ksp || !reason) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument");
  *reason = ksp->reason;
  return 0;
}
PetscErrorCode KSPConvergedReasonView(KSP ksp, void* viewer) {
  (void)viewer;
  if (!ksp) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null KSP");
  const bool conv = (int)ksp->reason > 0;
  printf("Linear solve %s due to %s iterations %d\n", conv ? "converged" : "did not converge",
         reason_name(ksp->reason), ksp->its);
  fflush(stdout);
  return 0;
}
PetscErrorCode KSPDestroy(KSP* ksp) {
  if (!ksp || !*ksp) return 0;
  delete *ksp;
  *ksp = nullptr;
  return 0;
}

// ------------------------------------------------------------------------------------------
// PreMixFEM_3D.h
int mkl_serv_intel_cpu_true() { return 1; }

PetscErrorCode PC_init(PCCtx* s_ctx, PetscScalar* dom, PetscInt* mesh) {
  if (!s_ctx || !dom || !mesh) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null argument to PC_init");
  // argument checks and option defaults of src/PreMixFEM_3D.c:1653-1705
  PetscCheck((dom[0] > 0.0 && dom[1] > 0.0 && dom[2] > 0.0), PETSC_COMM_WORLD, PETSC_ERR_ARG_WRONG,
             "Errors in dom(L, W, H)=[%.5f, %.5f, %.5f].\n", dom[0], dom[1], dom[2]);
  PetscCheck((mesh[0] > 0 && mesh[1] > 0 && mesh[2] > 0), PETSC_COMM_WORLD, PETSC_ERR_ARG_WRONG,
             "Errors in mesh(M, N, P)=[%d, %d, %d].\n", mesh[0], mesh[1], mesh[2]);
  memset(s_ctx, 0, sizeof(*s_ctx));
  pmf::Options o;
  std::string err;
  if (int e = pmf::options_from_db(g_db, &o, &err)) return SHIM_ERR(e, "%s", err.c_str());
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return SHIM_ERR(PETSC_ERR_LIB, "no CUDA device available");
  }
  s_ctx->L = dom[0];
  s_ctx->W = dom[1];
  s_ctx->H = dom[2];
  s_ctx->M = mesh[0];
  s_ctx->N = mesh[1];
  s_ctx->P = mesh[2];
  s_ctx->smoothing_iters_lv1 = o.si_lv1;
  s_ctx->smoothing_iters_lv2 = o.si_lv2;
  s_ctx->sub_domains = o.sd[0];
  {
    PetscInt sd_opt = 2;
    PetscCall(PetscOptionsGetInt(nullptr, nullptr, "-sd", &sd_opt, nullptr));
    if (sd_opt == 1)  // :1718-1721
      PetscCall(PetscPrintf(PETSC_COMM_WORLD,
                            "The subdomain may not be proper (too long/wide/high), reset sub_domains from %d to 2.\n",
                            sd_opt));
  }
  s_ctx->max_eigen_num_lv1 = o.en_lv1;
  s_ctx->max_eigen_num_lv2 = o.en_lv2;
  s_ctx->eigen_num_lv2 = 4;
  s_ctx->lv2_eigen_op = o.eg_op;
  s_ctx->eigen_bd_lv1 = o.eb_lv1 < 0.0 ? 1.0 / NIL : o.eb_lv1;
  s_ctx->eigen_bd_lv2 = o.eb_lv2 < 0.0 ? 1.0 / NIL : o.eb_lv2;
  s_ctx->use_W_cycle = o.use_W_cycle ? PETSC_TRUE : PETSC_FALSE;
  s_ctx->no_shift_A_cc = o.no_shift_A_cc ? PETSC_TRUE : PETSC_FALSE;
  s_ctx->use_full_Cholesky_lv1 = o.use_full_Cholesky_lv1 ? PETSC_TRUE : PETSC_FALSE;
  s_ctx->use_2level = o.use_2level ? PETSC_TRUE : PETSC_FALSE;
  s_ctx->H_x = dom[0] / (double)mesh[0];
  s_ctx->H_y = dom[1] / (double)mesh[1];
  s_ctx->H_z = dom[2] / (double)mesh[2];
  PetscCall(DMDACreate3d(PETSC_COMM_WORLD, DM_BOUNDARY_NONE, DM_BOUNDARY_NONE, DM_BOUNDARY_NONE, DMDA_STENCIL_STAR,
                         mesh[0], mesh[1], mesh[2], PETSC_DECIDE, PETSC_DECIDE, PETSC_DECIDE, 1, 1, nullptr, nullptr,
                         nullptr, &s_ctx->dm));
  try {
    s_ctx->dm->solver = new pmf::Solver(dom, mesh, o);
  } catch (const std::exception& ex) {
    DMDestroy(&s_ctx->dm);
    return SHIM_ERR(PETSC_ERR_LIB, "%s", ex.what());
  }
  // bookkeeping arrays, sized for every subdomain of every virtual rank
  const int nsub = o.sd[0] * o.sd[1] * o.sd[2] * o.vranks[0] * o.vranks[1] * o.vranks[2];
  s_ctx->ms_bases_c = (Vec*)calloc((size_t)o.en_lv1 * nsub, sizeof(Vec));
  s_ctx->ms_bases_cc = (Vec*)calloc((size_t)o.en_lv2, sizeof(Vec));
  s_ctx->ksp_lv1 = (KSP*)calloc((size_t)nsub, sizeof(KSP));
  PetscInt** starts[3] = {&s_ctx->coarse_startx, &s_ctx->coarse_starty, &s_ctx->coarse_startz};
  PetscInt** lens[3] = {&s_ctx->coarse_lenx, &s_ctx->coarse_leny, &s_ctx->coarse_lenz};
  for (int a = 0; a < 3; ++a) {
    const int cnt = o.sd[a] * o.vranks[a];
    PetscCall(PetscMalloc1(cnt, starts[a]));
    PetscCall(PetscMalloc1(cnt, lens[a]));
    // global starts/lengths of the subdomain slabs along this axis: the rank
    // split of the DMDA, then each rank's split into sd parts (:59-67)
    int pos = 0;
    for (int rk = 0; rk < o.vranks[a]; ++rk) {
      const int n = mesh[a] / o.vranks[a] + (mesh[a] % o.vranks[a] > rk ? 1 : 0);
      for (int i = 0; i < o.sd[a]; ++i) {
        const int len = n / o.sd[a] + (n % o.sd[a] > i ? 1 : 0);
        (*starts[a])[rk * o.sd[a] + i] = pos;
        (*lens[a])[rk * o.sd[a] + i] = len;
        pos += len;
      }
    }
  }
  PetscCall(PetscMalloc1(nsub, &s_ctx->eigen_num_lv1));
  PetscCall(PetscMalloc1(nsub, &s_ctx->eigen_max_lv1));
  PetscCall(PetscMalloc1(nsub, &s_ctx->eigen_min_lv1));
  for (int i = 0; i < nsub; ++i) {
    s_ctx->eigen_num_lv1[i] = 0;
    s_ctx->eigen_max_lv1[i] = s_ctx->eigen_min_lv1[i] = 0.0;
  }
  return 0;
}

PetscErrorCode PC_print_info(PCCtx* s_ctx) {
  if (!s_ctx || !s_ctx->dm || !s_ctx->dm->solver) return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "PC_init first");
  const pmf::Options& o = s_ctx->dm->solver->opt;
  PetscCall(PetscPrintf(PETSC_COMM_WORLD, "DIM=%d, M=%d, N=%d, P=%d.\n", 3, s_ctx->M, s_ctx->N, s_ctx->P));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD, "MPI Processes in each direction: X=%d, Y=%d, Z=%d.\n", o.vranks[0],
                        o.vranks[1], o.vranks[2]));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD,
                        "smoothing_iters_lv1=%d, smoothing_iters_lv2=%d, sub_domains=%d, lv2_eigen_op=%d\n",
                        s_ctx->smoothing_iters_lv1, s_ctx->smoothing_iters_lv2, s_ctx->sub_domains,
                        s_ctx->lv2_eigen_op));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD, "max_eigen_num_lv1=%d, eigen_bd_lv1=%.5E\n", s_ctx->max_eigen_num_lv1,
                        s_ctx->eigen_bd_lv1));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD, "max_eigen_num_lv2=%d, eigen_bd_lv2=%.5E\n", s_ctx->max_eigen_num_lv2,
                        s_ctx->eigen_bd_lv2));
  if (s_ctx->use_2level) PetscCall(PetscPrintf(PETSC_COMM_WORLD, "Only use the 2-level version!\n"));
  return 0;
}

static PetscErrorCode upload_kappa(PCCtx* s_ctx) {
  for (int i = 0; i < DIM; ++i)
    if (!s_ctx->kappa[i]) return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "s_ctx->kappa[%d] is not set", i);
  const PetscInt n = s_ctx->M * s_ctx->N * s_ctx->P;
  for (int i = 0; i < DIM; ++i)
    if (s_ctx->kappa[i]->n != n) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "kappa[%d] does not match the DMDA", i);
  pmf::Solver* s = s_ctx->dm->solver;
  return solver_call(s, s->set_kappa(s_ctx->kappa[0]->a, s_ctx->kappa[1]->a, s_ctx->kappa[2]->a, false));
}

PetscErrorCode PC_create_A(PCCtx* s_ctx, Mat* A) {
  if (!s_ctx || !A || !s_ctx->dm || !s_ctx->dm->solver)
    return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "PC_init must come before PC_create_A");
  PetscCall(upload_kappa(s_ctx));
  pmf::Solver* s = s_ctx->dm->solver;
  PetscCall(solver_call(s, s->assemble()));
  Mat m = new _p_Mat;
  m->dm = s_ctx->dm;
  *A = m;
  return 0;
}

PetscErrorCode _PC_setup(PCCtx* s_ctx) {
  if (!s_ctx || !s_ctx->dm || !s_ctx->dm->solver) return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "PC_init first");
  PetscCall(upload_kappa(s_ctx));
  pmf::Solver* s = s_ctx->dm->solver;
  PetscCall(solver_call(s, s->setup()));
  // eigenvalue bookkeeping of src/PreMixFEM_3D.c:367-383 and :1101-1115
  const int k = s->opt.en_lv1;
  for (int i = 0; i < s->nsub; ++i) {
    const int ki = s->ks[i];
    s_ctx->eigen_num_lv1[i] = ki;
    s_ctx->eigen_min_lv1[i] = s->eig1[(size_t)i * k];
    s_ctx->eigen_max_lv1[i] = s->eig1[(size_t)i * k + (ki > 0 ? ki - 1 : 0)];
  }
  const int k3 = s->ks3.empty() ? 0 : s->ks3[0];
  s_ctx->eigen_num_lv2 = k3;
  s_ctx->eigen_min_lv2 = s->eig3.empty() ? 0.0 : s->eig3[0];
  s_ctx->eigen_max_lv2 = s->eig3.empty() ? 0.0 : s->eig3[k3 > 0 ? k3 - 1 : 0];
  for (int i = 0; i < STAGE_SU; ++i) s_ctx->t_stages[i] = s->t_stages[i];
  return 0;
}

PetscErrorCode PC_setup(PC pc) {
  PetscLogDouble t;
  PetscCall(PetscTime(&t));
  PCCtx* s_ctx = nullptr;
  PetscCall(PCShellGetContext(pc, &s_ctx));
  if (!s_ctx) return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "PCSHELL context is not a PCCtx");
  PetscCall(_PC_setup(s_ctx));
  PetscCall(PetscTimeSubtract(&t));
  s_ctx->t_stages[STAGE_SU] -= t;
  return 0;
}

PetscErrorCode PC_apply_vec(PC pc, Vec x, Vec y) {
  PetscLogDouble t;
  PetscCall(PetscTime(&t));
  PCCtx* s_ctx = nullptr;
  PetscCall(PCShellGetContext(pc, &s_ctx));
  if (!s_ctx || !s_ctx->dm || !s_ctx->dm->solver)
    return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "PCSHELL context is not a PCCtx");
  PetscCall(same_size(x, y));
  if (x == y) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "x and y must be different vectors");
  pmf::Solver* s = s_ctx->dm->solver;
  PetscCall(solver_call(s, s->pc_apply(x->a, y->a, false)));
  for (int i = STAGE_AV_LV1; i <= STAGE_AV_LV3; ++i) s_ctx->t_stages[i] = s->t_stages[i];
  PetscCall(PetscTimeSubtract(&t));
  s_ctx->t_stages[STAGE_AV] -= t;
  return 0;
}

PetscErrorCode PC_get_range(const void* sendbuff, void* recvbuff, MPI_Datatype datatype) {
  // one process: the min and max over processes are the local value
  if (!sendbuff || !recvbuff) return SHIM_ERR(PETSC_ERR_ARG_WRONG, "null buffer");
  if (datatype == MPI_INT) {
    const PetscInt v = *(const PetscInt*)sendbuff;
    ((PetscInt*)recvbuff)[0] = v;
    ((PetscInt*)recvbuff)[1] = v;
  }
  if (datatype == MPI_DOUBLE) {
    const PetscScalar v = *(const PetscScalar*)sendbuff;
    ((PetscScalar*)recvbuff)[0] = v;
    ((PetscScalar*)recvbuff)[1] = v;
  }
  return 0;
}

PetscErrorCode PC_print_stat(PCCtx* s_ctx) {
  if (!s_ctx || !s_ctx->dm || !s_ctx->dm->solver) return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "PC_init first");
  pmf::Solver* s = s_ctx->dm->solver;
  if (!s->is_setup) return SHIM_ERR(PETSC_ERR_ARG_WRONGSTATE, "PC_setup has not run");
  // ranges over every subdomain and every virtual rank (src/PreMixFEM_3D.c:1954-1999)
  double mx1[2] = {0, 0}, mn1[2] = {0, 0};
  int num1[2] = {0, 0};
  for (int i = 0; i < s->nsub; ++i) {
    const double a = s_ctx->eigen_max_lv1[i], b = s_ctx->eigen_min_lv1[i];
    const int c = s_ctx->eigen_num_lv1[i];
    if (i == 0) {
      mx1[0] = mx1[1] = a;
      mn1[0] = mn1[1] = b;
      num1[0] = num1[1] = c;
    } else {
      mx1[0] = fmin(mx1[0], a);
      mx1[1] = fmax(mx1[1], a);
      mn1[0] = fmin(mn1[0], b);
      mn1[1] = fmax(mn1[1], b);
      num1[0] = std::min(num1[0], c);
      num1[1] = std::max(num1[1], c);
    }
  }
  double mx2[2] = {0, 0}, mn2[2] = {0, 0};
  int num2[2] = {0, 0}, size3 = 0;
  for (int r = 0; r < (int)s->ks3.size(); ++r) {
    const int k3 = s->ks3[r];
    const double a = s->eig3[(size_t)r * s->en2 + (k3 > 0 ? k3 - 1 : 0)], b = s->eig3[(size_t)r * s->en2];
    size3 += k3;
    if (r == 0) {
      mx2[0] = mx2[1] = a;
      mn2[0] = mn2[1] = b;
      num2[0] = num2[1] = k3;
    } else {
      mx2[0] = fmin(mx2[0], a);
      mx2[1] = fmax(mx2[1], a);
      mn2[0] = fmin(mn2[0], b);
      mn2[1] = fmax(mn2[1], b);
      num2[0] = std::min(num2[0], k3);
      num2[1] = std::max(num2[1], k3);
    }
  }
  const double* t = s_ctx->t_stages;
  PetscCall(PetscPrintf(PETSC_COMM_WORLD,
                        "eigen_max_lv1_range=[%.5E, %.5E], \teigen_min_lv1_range=[%.5E, %.5E], "
                        "\teigen_num_lv1_range=[%d, %d].\n",
                        mx1[0], mx1[1], mn1[0], mn1[1], num1[0], num1[1]));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD,
                        "eigen_max_lv2_range=[%.5E, %.5E], \teigen_min_lv2_range=[%.5E, %.5E], "
                        "\teigen_num_lv2_range=[%d, %d], \tsize_mat_lv3=%d.\n",
                        mx2[0], mx2[1], mn2[0], mn2[1], num2[0], num2[1], size3));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD,
                        "su_lv1=[%.5f, %.5f], \tsu_lv2_1=[%.5f, %.5f], \tsu_lv2_2=[%.5f, %.5f], \tsu_lv3_1=[%.5f, "
                        "%.5f], \tsu_lv3_2=[%.5f, %.5f], \tsu=[%.5f, %.5f].\n",
                        t[STAGE_SU_LV1], t[STAGE_SU_LV1], t[STAGE_SU_LV2_1], t[STAGE_SU_LV2_1], t[STAGE_SU_LV2_2],
                        t[STAGE_SU_LV2_2], t[STAGE_SU_LV3_1], t[STAGE_SU_LV3_1], t[STAGE_SU_LV3_2],
                        t[STAGE_SU_LV3_2], t[STAGE_SU], t[STAGE_SU]));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD,
                        "av_lv1=[%.5f, %.5f], \tav_lv2=[%.5f, %.5f], \tav_lv3=[%.5f, %.5f], \tav=[%.5f, %.5f].\n",
                        t[STAGE_AV_LV1], t[STAGE_AV_LV1], t[STAGE_AV_LV2], t[STAGE_AV_LV2], t[STAGE_AV_LV3],
                        t[STAGE_AV_LV3], t[STAGE_AV], t[STAGE_AV]));
  return 0;
}

PetscErrorCode PC_final_default(PCCtx* s_ctx) {
  if (!s_ctx) return 0;
  PetscCall(DMDestroy(&s_ctx->dm));
  free(s_ctx->ms_bases_c);
  free(s_ctx->ms_bases_cc);
  free(s_ctx->ksp_lv1);
  s_ctx->ms_bases_c = s_ctx->ms_bases_cc = nullptr;
  s_ctx->ksp_lv1 = nullptr;
  PetscCall(PetscFree(s_ctx->coarse_startx));
  PetscCall(PetscFree(s_ctx->coarse_starty));
  PetscCall(PetscFree(s_ctx->coarse_startz));
  PetscCall(PetscFree(s_ctx->coarse_lenx));
  PetscCall(PetscFree(s_ctx->coarse_leny));
  PetscCall(PetscFree(s_ctx->coarse_lenz));
  PetscCall(PetscFree(s_ctx->eigen_num_lv1));
  PetscCall(PetscFree(s_ctx->eigen_max_lv1));
  PetscCall(PetscFree(s_ctx->eigen_min_lv1));
  return 0;
}

// The multiscale bases and level solvers live in device memory owned by the
// DM's solver (the reference keeps them as Vec/KSP objects in s_ctx); freeing
// the DM releases them.
PetscErrorCode PC_final(PCCtx* s_ctx) { return PC_final_default(s_ctx); }

}  // extern "C"
