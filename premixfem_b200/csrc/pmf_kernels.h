// Host-side launchers for the B200 PreMixFEM kernels (internal interface).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "pmf_common.cuh"

namespace pmf {

// Number of kernels this library has launched (reported by bench and tests).
extern unsigned long long g_launches;
inline void note_launch() { __atomic_fetch_add(&g_launches, 1ull, __ATOMIC_RELAXED); }

// Scalars of the preconditioned CG loop, resident on the device so that an
// iteration needs no host round trip (PETSc KSPSolve_CG recurrences).
struct PcgState {
  double dp, ttol, beta, betaold, dpi, dpiold, alpha, rnorm0;
  // done: 0 running, 1 converged (residual test), 2 max_it, 3 indefinite, 4 nan/inf,
  // 5 converged because z.r = 0 (KSP_CONVERGED_ATOL)
  int its, max_it, first, done;
};

constexpr int kCellThreads = 256;
int cell_blocks(long long n);  // grid size for grid-stride cell loops (fixed per n)
int pcg_part_capacity(const Grid& g);  // partial slots the PCG step kernels may write (>= cell_blocks)

// ---- operator ----------------------------------------------------------------
struct AssembleArgs {
  Grid g;
  const double *kx, *ky, *kz;  // permeability per direction (device)
  double cx, cy, cz;           // |face|^2/|cell| per direction
  double dir_val[6];           // Dirichlet value per face (x-,x+,y-,y+,z-,z+)
  int dir_on[6];
  // a batch of problems: the problem table and the problem of each layer (-1: separator)
  const ProbInfo* probs = nullptr;
  const int* layer_prob = nullptr;
};
// a batch: zero permeability in the cells that belong to no problem
void launch_zero_padding(const Grid& g, const ProbInfo* probs, const int* layer_prob, double* kx, double* ky,
                         double* kz, cudaStream_t st);
void launch_assemble(const AssembleArgs& a, double* tx, double* ty, double* tz, double* diag, double* db,
                     double* bval, cudaStream_t st);
void launch_to_f32(const double* in, float* out, long long n, cudaStream_t st);
void launch_to_f64(const float* in, double* out, long long n, cudaStream_t st);

// y = A x (FP64 operator).
void launch_spmv(const Grid& g, const double* tx, const double* ty, const double* tz, const double* diag,
                 const double* x, double* y, cudaStream_t st);

// ---- PCG -----------------------------------------------------------------------
void launch_pcg_start(const Grid& g, const double* b, double* x, double* r, double* part, PcgState* s, double rtol,
                      double atol, int max_it, cudaStream_t st);
// beta = z.r from nparts per-block partials (written by the preconditioner's last kernel).
void launch_pcg_beta_fin(const double* part, int nparts, PcgState* s, cudaStream_t st);
// same, computing the partials itself
void launch_pcg_beta(const double* r, const double* z, long long n, double* part, PcgState* s, cudaStream_t st);
// constant null space: z <- z - mean(z), then beta = z.r (zpart: cell_blocks(n) scratch partials)
void launch_pcg_null_beta(double* z, const double* r, long long n, double* part, double* zpart, PcgState* s,
                          cudaStream_t st);
void launch_pcg_iter_a(const Grid& g, const double* tx, const double* ty, const double* tz, const double* diag,
                       const double* z, const double* pin, double* pout, double* w, double* part, PcgState* s,
                       cudaStream_t st, int variant = 0);
// The main kernel of launch_pcg_iter_a alone (no state update): variant 0 the
// 2.5-D march where the mesh allows it, 1 the grid-stride kernel.  Returns the
// number of partial sums written.
int launch_pcg_iter_a_main(const Grid& g, const double* tx, const double* ty, const double* tz, const double* diag,
                           const double* z, const double* pin, double* pout, double* w, double* part,
                           const PcgState* s, cudaStream_t st, int variant);
void launch_pcg_iter_b(long long n, double* x, double* r, const double* p, const double* w, double* part,
                       PcgState* s, cudaStream_t st);
void launch_dot(const double* a, const double* b, long long n, double* part, double* out, cudaStream_t st);

// ---- CG over a batch of problems (k_batch.cu): per-problem scalars, 2-D grids
// (blocks x problems); all_done is set when every problem has stopped
void launch_bpcg_start(const ProbInfo* probs, int nprob, const double* b, double* x, double* r, double* part,
                       PcgState* st, double rtol, double atol, int max_it, int* all_done, int nblk, cudaStream_t s);
void launch_bpcg_beta(const ProbInfo* probs, int nprob, const double* part, PcgState* st, cudaStream_t s);
void launch_bpcg_iter_a(const Grid& g, const ProbInfo* probs, const int* layer_prob, int nprob, const double* tx,
                        const double* ty, const double* tz, const double* diag, const double* z, const double* pin,
                        double* pout, double* w, double* part, PcgState* st, int nblk, cudaStream_t s);
void launch_bpcg_iter_b(const ProbInfo* probs, int nprob, double* x, double* r, const double* p, const double* w,
                        double* part, PcgState* st, int* all_done, int nblk, cudaStream_t s);

// ---- level 1 (IC(0) block solves) -------------------------------------------
void launch_ic_factor(const Grid& g, const SubInfo* subs, int nsub, int max_lines, const double* tx, const double* ty,
                      const double* tz, const double* diag, double* inv_d, int* bad, cudaStream_t st);

// out = yin + IC^-1 (x - A yin)   (yin may be null -> rhs = x).
// T: precision of the sweep; x is FP64 (the CG residual) or T; out is T or
// FP64 (final visit, with dot(x, out) per subdomain written to part).
template <typename T>
void launch_ic_apply(const Grid& g, const SubInfo* subs, int nsub, int max_lines, int max_cells, const T* tx,
                     const T* ty, const T* tz, const T* diag, const T* inv_d, const double* x, const T* yin,
                     T* out_t, double* out_d, double* part, const int* done, cudaStream_t st, int threads = 0);

// The same solve with the IC(0) factor in a subdomain-blocked copy,
// coef[coff[s] + cl] = {tx, ty, tz, 1/D} of the cells of s in local order
// (float4 / double4), staged by one TMA bulk copy per subdomain.  Needs every
// subdomain 16 cells wide with ny*nz <= 256; the result equals launch_ic_apply's
// up to the rounding of contracted multiply-adds.  *err is set if a CTA's copy
// did not complete within its wait limit.  threads: 256 or 512.
template <typename T>
void launch_pack_ic_coef(const Grid& g, const SubInfo* subs, int nsub, const long long* coff, const T* tx,
                         const T* ty, const T* tz, const T* inv, void* coef, cudaStream_t st);
size_t ic_blk_coef_bytes(int prec_bytes);
template <typename T>
size_t ic_blk_smem_bytes(int max_cells);
template <typename T>
void launch_ic_apply_blk(const Grid& g, const SubInfo* subs, int nsub, int max_cells, const long long* coff,
                         const void* coef, const T* tx, const T* ty, const T* tz, const T* diag, const double* x,
                         const T* yin, T* out_t, double* out_d, double* part, const int* done, int* err,
                         cudaStream_t st, int threads);
// The same solve with all of a CTA's global loads (x, y, the diagonal and the
// subdomain's face halo) issued in one unrolled pass before any is used, 512
// threads.  Needs the blocked kernel's shapes with ny <= 16 and nz <= 16.
template <typename T>
size_t ic_stg_smem_bytes(int max_cells);
template <typename T>
void launch_ic_apply_stg(const Grid& g, const SubInfo* subs, int nsub, int max_cells, const long long* coff,
                         const void* coef, const T* tx, const T* ty, const T* tz, const T* diag, const double* x,
                         const T* yin, T* out_t, double* out_d, double* part, const int* done, int* err,
                         cudaStream_t st);

// Exact level-1 solves (-use_full_Cholesky_lv1): banded Cholesky of every
// subdomain block in natural order, column j of L at band[boff[s] + j*band_ld(b)],
// b = nx*ny; bad counts non-positive pivots.
int band_ld_host(int b);
void launch_band_chol_factor(const Grid& g, const SubInfo* subs, int nsub, int max_b, const double* tx,
                             const double* ty, const double* tz, const double* diag, const long long* boff,
                             double* band, int* bad, cudaStream_t st);
// out = yin + (L L^T)^-1 (x - A yin), the same contract as launch_ic_apply.
template <typename T>
void launch_band_chol_apply(const Grid& g, const SubInfo* subs, int nsub, int max_cells, const T* tx, const T* ty,
                            const T* tz, const T* diag, const long long* boff, const T* band, const double* x,
                            const T* yin, T* out_t, double* out_d, double* part, const int* done, cudaStream_t st);

// c[s*kmax + j] = sum_{cells of s} phi[c*kmax + j] * (x - A y)[c]   (y may be null)
template <typename T>
void launch_resid_restrict(const Grid& g, const SubInfo* subs, int nsub, int kmax, const T* tx, const T* ty,
                           const T* tz, const T* diag, const T* phi, const double* x, const T* y, double* c,
                           const int* done, cudaStream_t st, int threads = 256);

// y[c] += sum_j phi[c*kmax + j] * Z[s*kmax + j]
template <typename T>
void launch_prolong(const Grid& g, const SubInfo* subs, int nsub, int kmax, const T* phi, const double* Z, T* y,
                    const int* done, cudaStream_t st, int threads = 256);

// ---- coarse (FP64) -------------------------------------------------------------
// Where each virtual rank's coarse data live: rank r owns subdomains
// first[r] .. first[r+1]-1 (contiguous), so nr_r = (first[r+1] - first[r]) x kmax
// coarse dofs starting at first[r] x kmax; its dense nr_r x nr_r blocks start
// at off2[r], its level-3 vectors (nr_r x en2) at offv[r], its level-3 work
// (3 x nr_r x p) at offw[r].  A grid of ranks of equal size is the special case
// first[r] = r spr, off2[r] = r nr^2 ...; a batch of problems has one rank per
// problem and ragged sizes.  All arrays are device arrays of nrank + 1 entries;
// dof_rank (nsub x kmax) maps a coarse dof to its rank.
struct RankLayout {
  const int* first = nullptr;
  const long long* off2 = nullptr;
  const long long* offv = nullptr;
  const long long* offw = nullptr;
  const int* dof_rank = nullptr;
  int kmax = 0;
};
void launch_block_gemv_r(const RankLayout& L, long long ncoarse, const double* inv, const double* in, double* out,
                         const int* done, cudaStream_t st);
void launch_lv3_restrict_r(const RankLayout& L, int nrank, int en2, const double* V, const double* c, double* d,
                           const int* done, cudaStream_t st);
void launch_lv3_prolong_r(const RankLayout& L, long long ncoarse, int en2, const double* V, const double* w,
                          double* dz, const int* done, cudaStream_t st);
void launch_assemble_dense_r(const SubInfo* subs, int nrank, const RankLayout& L, long long total, const double* blk,
                             const double* gface, int mode, double* dense, cudaStream_t st);
// dense[r] += mu (relative != 0: mu x max |diag| of the block) on the diagonal, one CTA per rank
void launch_add_diag_r(const RankLayout& L, int nrank, double* dense, double mu, int relative, cudaStream_t st);
// Gauss-Jordan inverses of the ragged blocks (the multi-CTA form of launch_spd_inverse)
void launch_spd_inverse_r(const RankLayout& L, int nrank, int nr_max, double* dense, double tol, int* nnull,
                          cudaStream_t st);
// out = alpha*v_in_out_base - A2 * v   where A2 is block sparse: blk[s][b][kmax][kmax],
// b = 0 diagonal, 1..6 couplings to nb[b-1].  If base is null the base term is 0.
void launch_a2_mult(const SubInfo* subs, int nsub, int kmax, const double* blk, const double* v, const double* base,
                    double* out, const int* done, cudaStream_t st);
// out[r][i] = sum_j inv[r][i][j] * in[r][j] for nrank dense blocks of size nr (batched GEMV).
void launch_block_gemv(int nrank, int nr, const double* inv, const double* in, double* out, int accumulate,
                       const int* done, cudaStream_t st);
// Level-3 restriction / prolongation with the per-rank eigenvector blocks V[r][nr][en2].
void launch_lv3_restrict(int nrank, int nr, int en2, const double* V, const double* c, double* d, const int* done,
                         cudaStream_t st);
void launch_lv3_prolong(int nrank, int nr, int en2, const double* V, const double* w, double* dz, const int* done,
                        cudaStream_t st);
void launch_axpy(long long n, double a, const double* x, double* y, const int* done, cudaStream_t st);
void launch_copy(long long n, const double* x, double* y, const int* done, cudaStream_t st);

// ---- coarse setup ----------------------------------------------------------------
template <typename T>
void launch_galerkin(const Grid& g, const SubInfo* subs, int nsub, int kmax, const double* tx, const double* ty,
                     const double* tz, const double* diag, const T* phi, double* blk, double* gface,
                     cudaStream_t st);
// dense per-rank matrices from the block-sparse coarse operator.
// mode 0: principal block of Phi^T A Phi (level 2); mode 1: rank-Neumann (level 3 eigen)
void launch_assemble_dense(const SubInfo* subs, int nsub, int nrank, int spr, int kmax, const double* blk,
                           const double* gface, int mode, double* dense, cudaStream_t st);
// In-place batched SPD inverse by Gauss-Jordan; pivots <= tol*max|diag| are null directions.
void launch_spd_inverse(int nb, int n, double* a, double tol, int* nnull, cudaStream_t st);

// ---- -use_2level: banded Cholesky of the global coarse matrix (k_coarse_band.cu) ----
struct CBandPlan {
  long long nc = 0;   // coarse unknowns (nsub x kmax)
  long long b = 0;    // half-bandwidth in subdomain-grid order
  int B = 0;          // tile bandwidth (64 x 64 tiles)
  int NS = 0;         // superblocks of B tiles
  long long NTp = 0;  // tiles per side, padded to NS x B
  std::vector<int> perm;  // grid-order dof -> natural coarse dof (s x kmax + j), -1 for padding
  size_t tile_bytes = 0, T_bytes = 0, X_bytes = 0;
};
// grid: subdomains per axis; returns 62 if the boxes do not form that grid
int cband_plan(const std::vector<SubInfo>& subs, const int grid[3], int kmax, CBandPlan* p);
// A2 (+ shift on the diagonal) -> tile-band Cholesky factor T and superblock inverses X; nullf
// (NTp x 64 ints) flags null pivots (<= tol x max|diag|), nnull counts them; scale: one device double
void launch_cband_factor(const SubInfo* subs, int kmax, const double* blk, const int* d_perm, const CBandPlan& p,
                         double shift, double tol, double* T, double* X, int* nullf, int* nnull, double* scale,
                         cudaStream_t st);
// out = A2^+ c (natural coarse order); v, y, t: work vectors of NTp x 64 doubles
void launch_cband_solve(const int* d_perm, const CBandPlan& p, const double* T, const double* X, const double* c,
                        double* out, double* v, double* y, double* t, double* part, const int* done,
                        cudaStream_t st);

// ---- eigen solvers -----------------------------------------------------------------
struct LobpcgArgs {
  Grid g;
  const SubInfo* subs;
  int nsub;
  int k;      // eigenpairs wanted (en_lv1)
  int m;      // block size (k + guard)
  int kmax;   // phi stride
  int eg_op;  // mass matrix variant
  int max_it;
  double tol;
  double rel_floor;  // > 0: residual test relative to max(|lambda_j|, rel_floor x lscale) instead of lscale
  double sigma_rel;  // IC(0) preconditioner shift, relative
  unsigned long long seed;
  const double *tx, *ty, *tz, *diag, *db;  // FP64 operator
  const double *kx, *ky, *kz;              // permeability (for the MOD/MEAN mass)
  double Hx, Hy, Hz, meas;
  const double* xinit;  // optional initial block (per cell, m values), may be null
  // optional per-subdomain initial columns from the learned network: patch
  // layout [s][16^3 voxels][16 channels], columns 0..xinit_k-1 used, the rest random
  const float* xinit_patch;
  int xinit_k;
  // optional subset of subdomains to solve: sub_list[0 .. *nlist-1] (device), may be null
  const int* sub_list;
  const int* nlist;
  // optional work queue (one device int, zeroed by the launcher): CTAs take the
  // next subdomain with atomicAdd instead of the fixed stride blockIdx.x + k*gridDim.x
  int* queue;
  // phase-batched solver: 0 = whole solve in this kernel (per-CTA work slab);
  // 1 = set-up only (mass, IC(0) pivots, initial block and Rayleigh-Ritz) into
  // the per-subdomain slab and state; 2 = final Rayleigh-Ritz and output from them
  int mode;
  int final_batched;    // batched solver: 1 = final Rayleigh-Ritz and output as phase kernels, 0 = mode 2
  int init_batched;     // batched solver: 1 = set-up (mass, IC(0), initial block, Rayleigh-Ritz) as phase kernels, 0 = mode 1
  unsigned char* slab;  // per-subdomain work slabs (modes 1, 2), stride slab_stride
  size_t slab_stride;
  void* state;          // per-subdomain EbState array (modes 1, 2)
  int dirichlet_mask;   // bit f set: face f (x-,x+,y-,y+,z-,z+) is a Dirichlet face
  const ProbInfo* probs = nullptr;  // a batch: per-problem cell size and Dirichlet faces (SubInfo::prob)
  int ld;               // column stride of the work block vectors (set by the launcher)
  int ldc;              // stride of the shared-memory sweep arrays (set by the launcher)
  int mb;               // vectors per shared-memory sweep (set by the launcher)
  long long* prof;      // optional: per-CTA clock64 totals of 8 phases (diagnostics), may be null
};
// Work buffer size in bytes for the LOBPCG kernel, per concurrently processed subdomain.
size_t lobpcg_work_bytes(int max_cells, int m, int prec_bytes);
// One persistent CTA per block; each handles subdomains blockIdx.x, +nblocks, ...
// ks[s] receives the adaptive eigen count (first j with lambda_j >= eb, else k).
// status[s]: 0 converged, 2 stopped at the rounding floor (within 100 x tol), 1 hit max_it.
// Requires ny*nz <= 256 and cells <= PMF_MAX_SUB_CELLS, m <= 10.
template <typename T>
void launch_lobpcg(const LobpcgArgs& a, int nblocks, void* work, T* phi, double* evals, int* iters, int* status,
                   int* ks, double eb, int max_cells, int max_lines, cudaStream_t st);

// Phase-batched LOBPCG: the same iteration as launch_lobpcg, but each phase
// (residual norms, convergence control, IC(0)-preconditioned directions,
// A-images, Grams, Rayleigh-Ritz, basis update) is its own launch over every
// active subdomain, with the block vectors of all subdomains resident in HBM.
struct EbBuffers {
  unsigned char* slab = nullptr;  // nsub x slab_stride
  size_t slab_stride = 0;
  void* state = nullptr;          // nsub EbState
  double* Ybuf = nullptr;         // nsub x 32 x 32 Rayleigh-Ritz coefficients
  double* gpart = nullptr;        // nsub x nchunk x 2 x 32 x 32 partial Grams
  double* rpart = nullptr;        // nsub x nchunk x LB_MM partial residual norms
  int* nactive = nullptr;         // device counter
  int* alist = nullptr;           // nsub: compacted list of subdomains still iterating
  unsigned long long* colcells = nullptr;  // device: sum of (basis columns x cells) over sub-iterations
  double* phase_ms = nullptr;     // host, optional: accumulated ms of resid+control, preconditioner,
                                  // Gram, Rayleigh-Ritz, update, A-images; [6] lockstep iterations
  int* h_nactive = nullptr;       // pinned host copy
  int nchunk = 0;
};
size_t lobpcg_batched_slab_bytes(int max_cells, int m, int prec_bytes);
size_t lobpcg_batched_state_bytes();
int lobpcg_batched_nchunk(int max_cells);
// list (device) / nlist (host): subdomains to solve, or nullptr for all a.nsub.
template <typename T>
int launch_lobpcg_batched(const LobpcgArgs& a, const EbBuffers& b, const int* list, int nlist, T* phi, double* evals,
                          int* iters, int* status, int* ks, double eb, int max_cells, int max_lines, cudaStream_t st);

// Level-3 eigenpairs: smallest en2 of dense symmetric A[r] (nr x nr), via subspace
// iteration with the inverse of (A + mu I) (given as inv) and Rayleigh-Ritz.
void launch_dense_smallest_eig(const RankLayout& L, int nrank, int nr_max, int en2, int p, const double* A,
                               const double* inv, double* V, double* evals, int* iters, double tol, int max_it,
                               double* work, cudaStream_t st);

}  // namespace pmf
