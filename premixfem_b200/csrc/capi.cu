// Flat C ABI (include/pmf_b200.h) over pmf::Solver.
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>

#include "../../include/pmf_b200.h"
#include "tune.h"
#include "solver.h"

struct pmf_solver {
  pmf::Solver* s;
};

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  fprintf(stderr, "[premixfem_b200] error %d: %s\n", code, msg.c_str());
  return code;
}
static int wrap(pmf_solver* h, int code) {
  if (code) return fail(code, h->s->err);
  return 0;
}

#define PMF_CHECK_HANDLE(h)                                        \
  do {                                                             \
    if (!(h) || !(h)->s) return fail(62, "null solver handle");    \
  } while (0)

// accessors for entry points defined in other translation units (noalloc.cu)
pmf::Solver* pmf_internal_solver(pmf_solver* h) { return h ? h->s : nullptr; }
int pmf_internal_fail(int code, const char* msg) { return fail(code, msg); }

extern "C" {

int pmf_create(const double dom[3], const int mesh[3], const char* options, pmf_solver** out) {
  if (!dom || !mesh || !out) return fail(62, "null argument to pmf_create");
  // PC_init argument checks (src/PreMixFEM_3D.c:1653-1654)
  if (!(dom[0] > 0.0 && dom[1] > 0.0 && dom[2] > 0.0)) return fail(62, "Errors in dom(L, W, H)");
  if (!(mesh[0] > 0 && mesh[1] > 0 && mesh[2] > 0)) return fail(62, "Errors in mesh(M, N, P)");
  // options first: their errors do not depend on a device
  pmf::OptionDB db;
  db.parse(options ? options : "");
  pmf::Options o;
  std::string err;
  if (int e = pmf::options_from_db(db, &o, &err)) return fail(e, err);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(76, "no CUDA device available");
  try {
    pmf_solver* h = new pmf_solver;
    h->s = new pmf::Solver(dom, mesh, o);
    *out = h;
  } catch (const std::exception& ex) {
    return fail(76, ex.what());
  }
  return 0;
}

int pmf_batch_create(int nprob, const double* dom, const int* mesh, const int* sd, const char* options,
                     pmf_solver** out) {
  if (nprob < 1 || !dom || !mesh || !sd || !out) return fail(62, "pmf_batch_create: bad argument");
  for (int q = 0; q < nprob; ++q) {
    if (!(dom[3 * q] > 0.0 && dom[3 * q + 1] > 0.0 && dom[3 * q + 2] > 0.0))
      return fail(62, "Errors in dom(L, W, H) of problem " + std::to_string(q));
    if (!(mesh[3 * q] > 0 && mesh[3 * q + 1] > 0 && mesh[3 * q + 2] > 0))
      return fail(62, "Errors in mesh(M, N, P) of problem " + std::to_string(q));
  }
  pmf::OptionDB db;
  db.parse(options ? options : "");
  pmf::Options o;
  std::string err;
  if (int e = pmf::options_from_db(db, &o, &err)) return fail(e, err);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(76, "no CUDA device available");
  try {
    pmf_solver* h = new pmf_solver;
    h->s = new pmf::Solver(nprob, dom, mesh, sd, o);
    *out = h;
  } catch (const std::exception& ex) {
    return fail(76, ex.what());
  }
  return 0;
}

int pmf_batch_info(pmf_solver* h, int shared_mesh[3], int* z0) {
  PMF_CHECK_HANDLE(h);
  pmf::Solver& s = *h->s;
  if (!s.nprob) return fail(73, "not a batch of problems");
  if (shared_mesh) {
    shared_mesh[0] = s.g.M;
    shared_mesh[1] = s.g.N;
    shared_mesh[2] = s.g.P;
  }
  if (z0)
    for (int q = 0; q < s.nprob; ++q) z0[q] = s.probs[q].z0;
  return 0;
}

int pmf_batch_set_dirichlet(pmf_solver* h, int q, int face, double value) {
  PMF_CHECK_HANDLE(h);
  return wrap(h, h->s->set_dirichlet_prob(q, face, value));
}

int pmf_batch_solve(pmf_solver* h, const double* b, double* x, int on_device, int* its, double* rnorm, int* reason) {
  PMF_CHECK_HANDLE(h);
  if (!b || !x) return fail(62, "null vector");
  return wrap(h, h->s->solve_batch(b, x, on_device != 0, its, rnorm, reason));
}

int pmf_destroy(pmf_solver* h) {
  if (!h) return 0;
  delete h->s;
  delete h;
  return 0;
}

int pmf_set_kappa(pmf_solver* h, const double* kx, const double* ky, const double* kz, int on_device) {
  PMF_CHECK_HANDLE(h);
  if (!kx) return fail(62, "kappa[0] is null");
  return wrap(h, h->s->set_kappa(kx, ky, kz, on_device != 0));
}

int pmf_set_dirichlet(pmf_solver* h, int face, double value) {
  PMF_CHECK_HANDLE(h);
  return wrap(h, h->s->set_dirichlet(face, value));
}

int pmf_setup(pmf_solver* h) {
  PMF_CHECK_HANDLE(h);
  return wrap(h, h->s->setup());
}

int pmf_rhs(pmf_solver* h, const double* source, double* rhs, int on_device) {
  PMF_CHECK_HANDLE(h);
  if (!source || !rhs) return fail(62, "null vector");
  return wrap(h, h->s->rhs(source, rhs, on_device != 0));
}

int pmf_apply_A(pmf_solver* h, const double* x, double* y, int on_device) {
  PMF_CHECK_HANDLE(h);
  if (!x || !y) return fail(62, "null vector");
  return wrap(h, h->s->apply_A(x, y, on_device != 0));
}

int pmf_pc_apply(pmf_solver* h, const double* x, double* y, int on_device) {
  PMF_CHECK_HANDLE(h);
  if (!x || !y) return fail(62, "null vector");
  return wrap(h, h->s->pc_apply(x, y, on_device != 0));
}

int pmf_solve(pmf_solver* h, const double* b, double* x, int on_device, int* its, double* rnorm, int* reason) {
  PMF_CHECK_HANDLE(h);
  if (!b || !x) return fail(62, "null vector");
  return wrap(h, h->s->solve(b, x, on_device != 0, its, rnorm, reason));
}

int pmf_profile_iteration(pmf_solver* h, int reps, double ms[8], int launches[8]) {
  PMF_CHECK_HANDLE(h);
  if (!ms || !launches || reps < 1) return fail(62, "pmf_profile_iteration: null output or reps < 1");
  return wrap(h, h->s->profile_iteration(reps, ms, launches));
}

int pmf_get_info(pmf_solver* h, int info[12]) {
  PMF_CHECK_HANDLE(h);
  pmf::Solver& s = *h->s;
  info[0] = (int)s.g.ncell;
  info[1] = s.nsub;
  info[2] = s.nrank;
  info[3] = s.spr;
  info[4] = s.kmax;
  info[5] = s.nr;
  info[6] = s.en2;
  info[7] = s.n3;
  info[8] = s.max_cells;
  info[9] = s.max_lines;
  info[10] = s.opt.precision;
  info[11] = s.is_setup ? 1 : 0;
  return 0;
}

int pmf_get_eigen_lv1(pmf_solver* h, double* evals, int* ks, int* iters, int* status) {
  PMF_CHECK_HANDLE(h);
  pmf::Solver& s = *h->s;
  if (!s.is_setup) return fail(73, "setup not done");
  if (evals) memcpy(evals, s.eig1.data(), sizeof(double) * s.eig1.size());
  if (ks) memcpy(ks, s.ks.data(), sizeof(int) * s.ks.size());
  if (iters) memcpy(iters, s.eig_iters.data(), sizeof(int) * s.eig_iters.size());
  if (status) memcpy(status, s.eig_status.data(), sizeof(int) * s.eig_status.size());
  return 0;
}

int pmf_get_eigen_lv2(pmf_solver* h, double* evals, int* ks, int* iters) {
  PMF_CHECK_HANDLE(h);
  pmf::Solver& s = *h->s;
  if (!s.is_setup) return fail(73, "setup not done");
  if (evals) memcpy(evals, s.eig3.data(), sizeof(double) * s.eig3.size());
  if (ks) memcpy(ks, s.ks3.data(), sizeof(int) * s.ks3.size());
  if (iters) memcpy(iters, s.l3_iters.data(), sizeof(int) * s.l3_iters.size());
  return 0;
}

int pmf_get_subdomains(pmf_solver* h, int* boxes, int* ranks) {
  PMF_CHECK_HANDLE(h);
  pmf::Solver& s = *h->s;
  if (s.subs.empty()) return fail(73, "partition not built (set kappa first)");
  for (int i = 0; i < s.nsub; ++i) {
    const pmf::SubInfo& S = s.subs[i];
    if (boxes) {
      int* b = boxes + 6 * i;
      b[0] = S.x0;
      b[1] = S.nx;
      b[2] = S.y0;
      b[3] = S.ny;
      b[4] = S.z0;
      b[5] = S.nz;
    }
    if (ranks) ranks[i] = S.rank;
  }
  return 0;
}

int pmf_get_phi(pmf_solver* h, double* out) {
  PMF_CHECK_HANDLE(h);
  pmf::Solver& s = *h->s;
  if (!s.is_setup) return fail(73, "setup not done");
  const size_t n = (size_t)s.g.ncell * s.kmax;
  if (s.opt.precision == 1) {
    double* tmp = nullptr;
    if (cudaMalloc(&tmp, n * 8) != cudaSuccess) return fail(76, "cudaMalloc");
    pmf::launch_to_f64((const float*)s.phi, tmp, (long long)n, s.st);
    cudaMemcpyAsync(out, tmp, n * 8, cudaMemcpyDeviceToHost, s.st);
    cudaStreamSynchronize(s.st);
    cudaFree(tmp);
  } else {
    cudaMemcpyAsync(out, s.phi, n * 8, cudaMemcpyDeviceToHost, s.st);
    cudaStreamSynchronize(s.st);
  }
  return 0;
}

int pmf_get_coarse_blocks(pmf_solver* h, double* out) {
  PMF_CHECK_HANDLE(h);
  pmf::Solver& s = *h->s;
  if (!s.is_setup) return fail(73, "setup not done");
  cudaMemcpy(out, s.blk, sizeof(double) * s.nsub * 7 * s.kmax * s.kmax, cudaMemcpyDeviceToHost);
  return 0;
}

int pmf_get_stages(pmf_solver* h, double t[10]) {
  PMF_CHECK_HANDLE(h);
  for (int i = 0; i < 10; ++i) t[i] = h->s->t_stages[i];
  return 0;
}

int pmf_get_timing(pmf_solver* h, double* setup_ms, double* solve_ms) {
  PMF_CHECK_HANDLE(h);
  if (setup_ms) *setup_ms = h->s->last_setup_ms;
  if (solve_ms) *solve_ms = h->s->last_solve_ms;
  return 0;
}

int pmf_get_eig_phases(pmf_solver* h, double ms[8], unsigned long long* colcells) {
  PMF_CHECK_HANDLE(h);
  if (ms)
    for (int i = 0; i < 8; ++i) ms[i] = h->s->eig_phase_ms[i];
  if (colcells) *colcells = h->s->eig_colcells;
  return 0;
}

int pmf_tune_report(char* buf, int len) {
  const std::string r = pmf::tune_report();
  if (buf && len > 0) {
    const int n = std::min<int>(len - 1, (int)r.size());
    memcpy(buf, r.data(), n);
    buf[n] = 0;
  }
  return (int)r.size();
}

unsigned long long pmf_launch_count(void) { return __atomic_load_n(&pmf::g_launches, __ATOMIC_RELAXED); }

const char* pmf_last_error(void) { return g_last_error.c_str(); }

int pmf_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

}  // extern "C"
