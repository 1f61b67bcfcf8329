// Host-side solver object behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "pmf_kernels.h"

namespace pmf {

// Preconditioner options; names follow PC_init (src/PreMixFEM_3D.c:1662-1705)
// plus the B200 extensions (-pmf_*).
struct Options {
  int sd[3] = {2, 2, 2};
  int vranks[3] = {1, 1, 1};
  int en_lv1 = 4, en_lv2 = 4;
  double eb_lv1 = -1.0, eb_lv2 = -1.0;
  int si_lv1 = 1, si_lv2 = 1;
  int eg_op = 0;
  bool use_W_cycle = false, no_shift_A_cc = false, use_full_Cholesky_lv1 = false, use_2level = false;
  bool null_space = false;  // -ksp_constant_null_space: the constant is the operator's null space
  int precision = 0;  // 0 plain FP64, 1 FP32 preconditioner inside FP64 PCG
  double rtol = 1e-8;
  double atol = 1e-50;  // KSP abstol (PETSc default)
  int max_it = 10000;
  int eig_max_it = 300;
  double eig_tol = -1.0;  // < 0: 1e-8 for the FP64 setup, 1e-6 for the FP32 setup
  double eig_sigma = 1e-2;
  int eig_guard = 2;
  int l3_max_it = 500;
  double l3_tol = 1e-10;
  unsigned long long seed = 20240611ull;
  int pcg_chunk = 4;
  int pcg_graph = 1;  // replay each chunk of PCG iterations as one CUDA graph
  int eig_final = 1;  // batched eigensolver: final Rayleigh-Ritz and output as phase kernels (0: one persistent launch)
  double eig_rel_floor = 0.0;  // > 0: eigen residual test relative to max(|lambda|, floor x lscale)
  int eig_init = 0;   // batched eigensolver: 1 = set-up as phase kernels, 0 = one persistent launch
  int autotune = -1;  // launch-shape tuning: 1 on, 0 off, -1 the process default (PMF_AUTOTUNE)
  int eig_ctas = 0;  // persistent CTAs of the batched eigensolver (0: one per SM)
  int eig_batched = 1;  // 1: phase-batched LOBPCG (one launch per phase), 0: one persistent launch
  int eig_profile = 0;  // 1: time each phase of the batched eigensolver (pmf_get_eig_phases)
  bool eig_require_converged = false;  // a local eigensolve that hits eig_max_it fails the set-up (error 83)
  int lv1_kernel = 0;  // level-1 solve kernel: 0 the tuner's choice, 1 natural-order, 2 subdomain-blocked,
                       // 3 subdomain-blocked with all global loads staged up front
  int eig_precision = -1;  // local eigensolver vectors: -1 as the preconditioner, 0 FP64, 1 FP32 (mixed only)
  // learned initial blocks for the local eigensolves (-pmf_learned <weights>):
  // LOBPCG starts from the network's output and may take learned_its
  // iterations; subdomains that have not converged by then are solved again
  // from a random start with the full iteration budget
  std::string learned_path;
  int learned_its = 60;
  double learned_tol = -1.0;  // Ritz-residual gate of the learned start (< 0: the eigensolver's own tolerance)
};

// PETSc-style options database ("-name value" pairs); flags carry an empty value.
struct OptionDB {
  std::map<std::string, std::string> kv;
  void parse(const std::string& s);
  bool has(const char* name) const { return kv.count(name) > 0; }
  bool get_int(const char* name, int* v) const;
  bool get_real(const char* name, double* v) const;
  bool get_ints(const char* name, int* v, int n) const;  // "a,b,c"
};
int options_from_db(const OptionDB& db, Options* o, std::string* err);

enum Stage {
  ST_SU_LV1 = 0,
  ST_SU_LV2_1,
  ST_SU_LV2_2,
  ST_SU_LV3_1,
  ST_SU_LV3_2,
  ST_AV_LV1,
  ST_AV_LV2,
  ST_AV_LV3,
  ST_SU,
  ST_AV,
  ST_COUNT
};

class Net;

class Solver {
 public:
  Solver(const double dom[3], const int mesh[3], const Options& o);
  // a batch of problems on one shared mesh (pmf_batch_create)
  Solver(int nprob, const double* doms, const int* meshes, const int* sds, const Options& o);
  ~Solver();

  int set_kappa(const double* kx, const double* ky, const double* kz, bool on_device);
  int set_dirichlet(int face, double value);
  int assemble();  // operator only (PC_create_A); setup() assembles as well
  int setup();
  int rhs(const double* source, double* out, bool on_device);
  int apply_A(const double* x, double* y, bool on_device);
  int pc_apply(const double* x, double* y, bool on_device);
  int solve(const double* b, double* x, bool on_device, int* its, double* rnorm, int* reason);

  // introspection for tests and stats
  Grid g;
  double dom[3], H[3];
  Options opt;
  cudaStream_t st = nullptr;
  std::vector<SubInfo> subs;
  int nsub = 0, nrank = 0, spr = 0, kmax = 0, max_cells = 0, max_lines = 0, nr = 0, en2 = 0, n3 = 0;
  int rank_grid[3];
  bool is_setup = false;
  std::vector<double> eig1, eig3;  // per subdomain k values / per rank en2 values
  std::vector<int> ks, ks3, eig_iters, eig_status, l3_iters;
  double t_stages[ST_COUNT] = {0};
  std::string err;

  // device data
  SubInfo* d_subs = nullptr;
  double *kx = nullptr, *ky = nullptr, *kz = nullptr;
  double *tx = nullptr, *ty = nullptr, *tz = nullptr, *diag = nullptr, *db = nullptr, *bval = nullptr;
  float *tx32 = nullptr, *ty32 = nullptr, *tz32 = nullptr, *diag32 = nullptr, *inv32 = nullptr;
  double* inv64 = nullptr;
  // -use_full_Cholesky_lv1: banded Cholesky factors of the subdomain blocks
  long long* d_boff = nullptr;
  double* band64 = nullptr;
  float* band32 = nullptr;
  long long band_len = 0;
  void* phi = nullptr;
  double *blk = nullptr, *gface = nullptr, *A2inv = nullptr, *AN = nullptr, *ANinv = nullptr, *V3 = nullptr,
         *A3inv = nullptr, *d_eig1 = nullptr, *d_eig3 = nullptr;
  int *d_ks = nullptr, *d_iters = nullptr, *d_status = nullptr, *d_l3it = nullptr, *d_flag = nullptr;
  int* d_rank_nb = nullptr;
  bool coarse_ok = false;  // the level-2/3 arrays above are allocated
  // where each virtual rank's coarse data live (pmf_kernels.h RankLayout);
  // rank_first is filled by the partition, the rest by rank_layout()
  std::vector<int> rank_first;  // nrank + 1
  bool ragged = false;          // ranks of different sizes (a batch of problems)
  long long tot2 = 0, totv = 0, totw = 0;
  int nr_min = 0, l3p = 0;
  RankLayout rl;
  int* d_rl_first = nullptr;
  long long* d_rl_off = nullptr;  // off2, offv, offw: 3 x (nrank + 1)
  int* d_rl_dof_rank = nullptr;
  void rank_sizes();   // host: nr, nr_min, en2, n3, l3p, tot2, totv, totw from rank_first
  int rank_layout();   // device copies of the layout
  // a batch of problems (0: one problem)
  int nprob = 0;
  std::vector<ProbInfo> probs;
  std::vector<int> bsd, layer_prob;
  ProbInfo* d_probs = nullptr;
  int* d_layer_prob = nullptr;
  int build_partition_batch();
  int partition_checks();
  int set_dirichlet_prob(int q, int face, double value);
  int upload_probs();
  // CG over the batch: one PCG per problem, one set of launches for all
  int solve_batch(const double* b, double* x, bool on_device, int* its, double* rnorm, int* reason);
  PcgState* bstate = nullptr;    // device, per problem
  PcgState* h_bstate = nullptr;  // pinned copy
  int* d_all_done = nullptr;
  int* h_all_done = nullptr;     // pinned
  cudaGraphExec_t bpcg_exec = nullptr;
  const double* bpcg_graph_x = nullptr;
  unsigned long long bpcg_graph_kernels = 0;
  int bpcg_blocks() const { return 32; }
  void* eig_work = nullptr;
  size_t eig_work_bytes = 0;
  double *c = nullptr, *dz = nullptr, *Zacc = nullptr, *d3 = nullptr, *w3 = nullptr;
  void *y0 = nullptr, *y1 = nullptr;
  double *vb = nullptr, *vx = nullptr, *r = nullptr, *z = nullptr, *p0 = nullptr, *p1 = nullptr, *w = nullptr,
         *part = nullptr;
  double* zpart = nullptr;  // tail of part: per-block sums of z for the constant null space
  PcgState* state = nullptr;
  PcgState* h_state = nullptr;  // pinned
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  int check(cudaError_t e, const char* what);
  int dalloc(void** p, size_t bytes, const char* what);
  int build_partition();
  int alloc_fine();
  void assemble_launch();
  template <typename T>
  void apply_impl(const double* x, double* out, double* partial, const int* done);
  void apply(const double* x, double* out, double* partial, const int* done);
  std::vector<int> schedule() const;
  int dir_on_[6] = {0, 0, 0, 0, 0, 0};
  double dir_val_[6] = {0, 0, 0, 0, 0, 0};
  double last_setup_ms = 0, last_solve_ms = 0;
  int last_its = 0;
  // learned set-up
  Net* net = nullptr;
  void* net_x = nullptr;  // BF16 feature patches of one chunk of subdomains
  float* net_y = nullptr;  // network output for every subdomain [nsub][4096][16]
  int* d_queue = nullptr;
  EbBuffers eb;  // phase-batched eigensolver storage
  double eig_phase_ms[8] = {0};
  cudaGraphExec_t pcg_exec = nullptr;  // one chunk of PCG iterations
  const double* pcg_graph_x = nullptr;
  bool pcg_graph_ns = false;  // the null-space setting the graph was captured with
  unsigned long long pcg_graph_kernels = 0;
  unsigned long long eig_colcells = 0;
  int alloc_eb(int m, bool mixed);
  int setup_band_cholesky(bool mixed);
  template <typename T>
  void tune_pc();
  int ic_threads = 0, rr_threads = 256, pr_threads = 256, pcga_variant = 0;  // tuned launch shapes
  // level-1 solve with the subdomain-blocked IC(0) factor (k_ic_apply_blk)
  bool ic_blk_ok = false;  // every subdomain fits the blocked kernel
  bool ic_stg_ok = false;  // ... and its staged form (k_ic_apply_stg: ny, nz <= 16)
  // per visit kind (0: first visit, no iterate; 1: visits with an iterate):
  // 0 natural-order kernel, 1 blocked kernel, 2 its staged form (tuner's
  // choice), and the blocked kernel's threads
  int ic_variant[2] = {0, 0}, ic_blk_threads[2] = {512, 512};
  long long* d_coff = nullptr;  // per subdomain: first cell in the blocked arrays
  void* ic_coef = nullptr;      // blocked {tx, ty, tz, 1/D} (precision of the preconditioner)
  int* d_kerr = nullptr;        // set by a kernel whose bounded wait ran out
  int check_kernel_flag(const char* what);
  int setup_ic_blocked(bool mixed);
  template <typename T>
  void launch_lv1(const double* x, const T* yin, T* out_t, double* out_d, double* partial, const int* done);
  int run_eigen(LobpcgArgs& la, const int* list, int nlist, int eig_blocks, double eb1);
  // the local eigensolves run on FP32 vectors (the mixed form's default)
  bool eig32() const { return opt.precision == 1 && opt.eig_precision != 0; }
  double* phi64 = nullptr;  // FP64 eigensolver output of the mixed form with -pmf_eig_precision fp64
  double* l3work = nullptr;  // level-3 subspace-iteration blocks
  int* d_ks3 = nullptr;
  // -use_2level: banded Cholesky of the global coarse matrix (k_coarse_band.cu)
  CBandPlan cband;
  double *cb_T = nullptr, *cb_X = nullptr, *cb_v = nullptr, *cb_y = nullptr, *cb_t = nullptr, *cb_scale = nullptr;
  double* cb_part = nullptr;  // column partial sums of the banded backward solve (B x B x 64)
  int *cb_perm = nullptr, *cb_null = nullptr;
  int setup_two_level();
  int *d_fail_list = nullptr, *d_fail_count = nullptr, *d_iters_learned = nullptr, *d_status_learned = nullptr;
  int learned_used = 0, learned_fallbacks = 0;
  long long learned_iters = 0, fallback_iters = 0;
  double net_ms = 0.0;
  int run_learned_eigen(LobpcgArgs& la, int eig_blocks, double eb1);
  int nparts_apply() const { return nsub; }
  // Per-kernel-class device time of one PCG iteration (profile_iteration):
  // while prof_on, apply_impl records an event after each launch group,
  // tagged with its class (PROF_* below).
  enum { PROF_LV1_FIRST = 0, PROF_LV1_Y, PROF_RESTRICT, PROF_COARSE, PROF_PROLONG, PROF_CG_A, PROF_CG_B, PROF_BETA,
         PROF_SLOTS };
  bool prof_on = false;
  int prof_n = 0;
  cudaEvent_t prof_ev[64] = {};
  int prof_slot[64] = {};
  void prof_mark(int slot);
  int profile_iteration(int reps, double ms[PROF_SLOTS], int launches[PROF_SLOTS]);
};

}  // namespace pmf
