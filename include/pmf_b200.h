/*
 * pmf_b200.h -- flat C ABI of the B200 PreMixFEM solver library
 * (libpremixfem_b200.so).  Plain pointers and sizes only; every function
 * returns 0 on success or a PETSc-style error code (62 bad argument, 73 wrong
 * state, 56 unsupported, 71 zero pivot, 76 CUDA/library failure, 83 a local
 * eigensolve did not converge) and leaves a message for pmf_last_error().
 *
 * Arrays are float64, natural order with x fastest (cell id
 * (ez*N + ey)*M + ex), the DMDA ordering the reference uses.  "on_device"
 * selects whether array arguments are device (CUDA) or host pointers.
 *
 * This ABI is what a foreign-function binding of the reference's solve path
 * would call (a ctypes binding, for instance); the PETSc-style drop-in header
 * PreMixFEM_3D.h is implemented on top of it.  Mapping to the
 * reference interface (src/PreMixFEM_3D.h of Laphet/PreMixFEM):
 *   pmf_create        <- PC_init            (src/PreMixFEM_3D.h:47, src/PreMixFEM_3D.c:1650-1741)
 *   pmf_set_kappa     <- caller fills PCCtx.kappa[3] (src/PreMixFEM_3D.h:34; src/Expe_scal.c:11-42)
 *   pmf_set_dirichlet <- (extension: Dirichlet faces; the reference is pure Neumann)
 *   pmf_apply_A       <- MatMult of the matrix built by PC_create_A (src/PreMixFEM_3D.h:55, .c:1757-1824)
 *   pmf_setup         <- PC_setup / _PC_setup (src/PreMixFEM_3D.h:53, .c:1392-1427, 1826-1838)
 *   pmf_pc_apply      <- PC_apply_vec       (src/PreMixFEM_3D.h:57, .c:1840-1936)
 *   pmf_solve         <- KSPSolve with KSPCG + the PCSHELL above (src/Expe_scal.c:100-119)
 *   pmf_get_stages    <- PCCtx.t_stages / PC_print_stat (src/PreMixFEM_3D.h:42, .c:1954-1999)
 *   pmf_get_eigen_*   <- PCCtx.eigen_{min,max,num}_lv{1,2} (src/PreMixFEM_3D.h:40-41)
 *   pmf_destroy       <- PC_final / PC_final_default (src/PreMixFEM_3D.h:63-65, .c:2001-2046)
 */
#ifndef PMF_B200_H
#define PMF_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pmf_solver pmf_solver;

/* Options use the reference's PETSc option names: -sd, -en_lv1, -en_lv2,
 * -eb_lv1, -eb_lv2, -si_lv1, -si_lv2, -eg_op, -use_W_cycle, -no_shift_A_cc,
 * -use_full_Cholesky_lv1 (banded Cholesky local solves), -use_2level,
 * -ksp_rtol, -ksp_max_it, -ksp_constant_null_space (PETSc's: the constant
 * vector is the operator's null space, removed from every preconditioned
 * residual of the CG solve; for operators with no Dirichlet face); B200
 * extensions: -pmf_sd sx,sy,sz (subdomains per
 * rank and axis), -pmf_vranks px,py,pz (virtual DMDA process grid),
 * -pmf_precision fp64|mixed, -pmf_eig_tol, -pmf_eig_max_it (a local eigensolve
 * that spends it keeps its last Ritz block and reports status 1; with
 * -pmf_eig_require_converged pmf_setup fails with 83 instead, as the
 * reference's SLEPc check does), -pmf_learned
 * <weights file> (learned initial blocks for the local eigensolves),
 * -pmf_learned_its N and -pmf_learned_tol t (a subdomain whose LOBPCG from the
 * learned start has not reached relative residual t within N iterations is
 * solved again from a random start at the normal tolerance; defaults 60 and
 * the eigensolver's own tolerance, so a learned start is held to the same
 * accuracy as a random one; t can only loosen it), -pmf_eig_batched 0|1 and
 * -pmf_eig_final 0|1 (phase-batched
 * eigensolver and its batched final phase, both on by default),
 * -pmf_eig_init 0|1 (set-up phase as batched kernels, off by default),
 * -pmf_eig_rel_floor f (0 <= f < 1; > 0: the local eigensolves stop when
 * ||r_j||_{M^-1} <= tol x max(|lambda_j|, f x lscale), an eigenvalue-relative
 * test, instead of tol x lscale with lscale = max diag(A_N)/M; experimental,
 * off by default),
 * -pmf_eig_profile 1 (per-phase timing, pmf_get_eig_phases), -pmf_pcg_graph
 * 0|1 (PCG iterations replayed as CUDA graphs, on by default), -pmf_autotune
 * 0|1 (launch-shape tuning, on by default; pmf_tune_report), -pmf_lv1_kernel
 * auto|natural|blocked|staged (level-1 solve kernel: the tuner's choice, the
 * natural-order kernel, the kernel that stages each subdomain's IC(0) factor
 * with one TMA bulk copy, which needs every subdomain 16 cells wide in x with
 * x0 and M multiples of 4, or that kernel with all of its other global loads
 * issued in one pass up front, which also needs ny <= 16 and nz <= 16; they
 * agree up to the rounding of contracted multiply-adds). */
int pmf_create(const double dom[3], const int mesh[3], const char* options, pmf_solver** out);
int pmf_destroy(pmf_solver* s);

int pmf_set_kappa(pmf_solver* s, const double* kx, const double* ky, const double* kz, int on_device);
/* face: 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+ */
int pmf_set_dirichlet(pmf_solver* s, int face, double value);
int pmf_setup(pmf_solver* s);

/* rhs = source + Dirichlet boundary contributions (needs pmf_setup). */
int pmf_rhs(pmf_solver* s, const double* source, double* rhs, int on_device);
int pmf_apply_A(pmf_solver* s, const double* x, double* y, int on_device);
int pmf_pc_apply(pmf_solver* s, const double* x, double* y, int on_device);
/* reason: 1 converged (residual test), 2 max_it, 3 indefinite, 4 nan/inf, 5 converged because the
 * preconditioned residual's dot z.r is exactly zero (PETSc's KSP_CONVERGED_ATOL for KSPCG) */
int pmf_solve(pmf_solver* s, const double* b, double* x, int on_device, int* its, double* rnorm, int* reason);

/* Device time of the kernels of one PCG iteration by class, after pmf_setup (and normally a
 * pmf_solve, whose final residual is the input): the iteration's launches run `reps` times outside
 * any CUDA graph with an event after each launch group, on scratch vectors (the solver's last
 * solution and residual are kept; its CG scalars are not).  ms[c] = mean device milliseconds per
 * iteration, launches[c] = launch groups per iteration, for the classes
 *   0 level-1 first visit (IC(0) sweeps of the residual), 1 level-1 visits with an iterate
 *   (r - A y, sweeps, y +=; the last one writes the FP64 result and the z.r partials),
 *   2 residual + level-2 restriction, 3 coarse solves (levels 2 and 3), 4 prolongation,
 *   5 CG p-update + A p, 6 CG x/r update + residual norm, 7 beta = z.r.
 * No counterpart in the reference (PETSc's -log_view plays this role there). */
int pmf_profile_iteration(pmf_solver* s, int reps, double ms[8], int launches[8]);

/*
 * A batch of independent problems solved together (many small problems of
 * different sizes; the reference solves one problem per run).  Problem q has
 * dom[3q..3q+2], mesh[3q..3q+2] and sd[3q..3q+2] subdomains per axis (one
 * virtual rank per problem: its level 2 is its whole coarse space).  The
 * problems share one mesh (pmf_batch_info: max M x max N x sum(P + 1) cells;
 * problem q fills x < M_q, y < N_q of the layers z0[q] .. z0[q] + P_q - 1,
 * the rest is zero-permeability padding); pmf_set_kappa, pmf_setup, pmf_rhs
 * and the pmf_get_* queries work on that shared layout.  Every set-up phase
 * runs one launch over the subdomains of all problems.  pmf_batch_solve runs
 * one PCG per problem (its, rnorm, reason: nprob entries each), all of them
 * in one set of launches per iteration.  -pmf_learned, -use_2level and
 * -ksp_constant_null_space are not available for batches (56); pmf_solve and
 * pmf_set_dirichlet return 73 on a batch.
 */
int pmf_batch_create(int nprob, const double* dom, const int* mesh, const int* sd, const char* options,
                     pmf_solver** out);
int pmf_batch_info(pmf_solver* s, int shared_mesh[3], int* z0);
int pmf_batch_set_dirichlet(pmf_solver* s, int q, int face, double value);
int pmf_batch_solve(pmf_solver* s, const double* b, double* x, int on_device, int* its, double* rnorm, int* reason);

/* info[0..11] = ncell_lo32, nsub, nrank, subdomains_per_rank, kmax, nr, en_lv2, n3,
 *               max_cells, max_lines, precision, is_setup */
int pmf_get_info(pmf_solver* s, int info[12]);
int pmf_get_eigen_lv1(pmf_solver* s, double* evals, int* ks, int* iters, int* status);
int pmf_get_eigen_lv2(pmf_solver* s, double* evals, int* ks, int* iters);
/* subdomain boxes: 6 ints per subdomain (x0, nx, y0, ny, z0, nz) and its rank */
int pmf_get_subdomains(pmf_solver* s, int* boxes, int* ranks);
/* basis Phi, ncell * kmax values (cell-major), converted to float64 */
int pmf_get_phi(pmf_solver* s, double* out);
/* Galerkin blocks, nsub * 7 * kmax * kmax (diagonal, x-, x+, y-, y+, z-, z+) */
int pmf_get_coarse_blocks(pmf_solver* s, double* out);
/* t[10]: su_lv1, su_lv2_1, su_lv2_2, su_lv3_1, su_lv3_2, av_lv1, av_lv2, av_lv3, su, av (seconds) */
int pmf_get_stages(pmf_solver* s, double t[10]);
/* last setup and solve time measured with CUDA events on the solver stream (ms) */
int pmf_get_timing(pmf_solver* s, double* setup_ms, double* solve_ms);

/*
 * Learned set-up (no counterpart in the reference, whose local eigensolves
 * always start from SLEPc's default vectors).  A 3-D convolutional
 * encoder-decoder maps each subdomain's log-permeability patch (16^3, zero
 * padded) to k initial vectors for LOBPCG.  All array arguments are device
 * memory, work runs on the legacy default stream; feats are BF16
 * [nsub][4096][16], V are FP32 [nsub][4096][k], M FP32 [nsub][4096], network
 * outputs y and gradients dy FP32 [B][4096][16].
 */
typedef struct pmf_net pmf_net;
int pmf_net_create(unsigned long long seed, pmf_net** out);   /* random (He) weights */
int pmf_net_load(const char* path, pmf_net** out);
int pmf_net_save(pmf_net* net, const char* path);
int pmf_net_destroy(pmf_net* net);
int pmf_net_params(pmf_net* net);                              /* parameter count */
/* info: type (0 conv3, 1 down2, 2 up2, 3 conv1), cin, cout, s_in, s_out, taps */
int pmf_net_layer_info(int layer, int info[6]);
int pmf_net_forward(pmf_net* net, const void* x, int B, float* y);
int pmf_net_backward(pmf_net* net, const float* dy, int B);   /* after pmf_net_forward of the same batch */
int pmf_net_adam(pmf_net* net, float lr, float beta1, float beta2, float eps, float weight_decay);
/* FP32 weights W[tap][cin][cout] and biases of one layer (host memory) */
int pmf_net_get_weights(pmf_net* net, int layer, float* w, float* b);
int pmf_net_set_weights(pmf_net* net, int layer, const float* w, const float* b);
int pmf_net_get_grads(pmf_net* net, int layer, float* gw, float* gb);
/* subspace loss per sample: loss[b] = ||V - Y C||_M^2 / k with C = (Y^T M Y)^-1 Y^T M V, and dL/dy
 * of the batch mean */
int pmf_net_loss(const float* y, const float* V, const float* M, int B, int k, float* loss, float* dy);
/* after pmf_setup: network inputs of every subdomain and, as training targets, its local
 * eigenvectors and mass diagonal (any of the three pointers may be NULL) */
int pmf_learned_patches(pmf_solver* s, void* feats, float* V, float* M);
/* stats: learned start used, subdomains that fell back, LOBPCG iterations from the learned start,
 * iterations of the fallbacks; net_ms: network inference time of the last set-up */
int pmf_get_learned_stats(pmf_solver* s, long long stats[4], double* net_ms);

/*
 * pmf_residual_noalloc -- has no counterpart in the reference (its residual is
 * a MatMult into a Vec it allocates, then VecAXPY and VecNorm).
 *
 * r = b - A x and rnorm[0] = ||r||_2 for DEVICE vectors b, x, r and a DEVICE
 * scalar rnorm, enqueued on `stream` (a cudaStream_t; NULL = the legacy
 * default stream); the call returns without waiting.  It allocates nothing,
 * host or device, on its success path: the reduction scratch is a static
 * device array inside the library.  For callers that cannot allocate at that
 * point: a device pool that owns all free memory, a per-iteration monitor
 * where cudaMalloc would synchronise the device, or a fixed launch sequence
 * that must not change between recordings.
 *   - meshes of more than PMF_NOALLOC_MAX_CELLS cells are rejected (error 62);
 *   - the operator must be assembled (pmf_setup done; else error 73), and the
 *     current device must be the solver's (else error 62);
 *   - the first call on each device resolves and zeroes the scratch (with
 *     cudaGetSymbolAddress and cudaMemset, synchronising the device): make that
 *     first call before any stream capture begins;
 *   - the scratch's ticket counter must be zero when a call starts: it is
 *     zero when the library's module loads, the first call on each device
 *     zeroes it again, and every completed call leaves it at zero;
 *   - all calls on one device share the scratch: overlapping calls (two
 *     streams, two threads) race and return wrong results; serialise them.
 */
#define PMF_NOALLOC_MAX_BLOCKS 16384
#define PMF_NOALLOC_MAX_CELLS 33554432LL /* PMF_NOALLOC_MAX_BLOCKS x 2048 cells */
int pmf_residual_noalloc(pmf_solver* s, const double* b, const double* x, double* r, double* rnorm, void* stream);

/* Phase-batched local eigensolver of the last pmf_setup (option -pmf_eig_profile 1 enables the
 * timing): ms[0..5] device ms of residual norms + control, IC(0)-preconditioned directions, Grams,
 * Rayleigh-Ritz, basis update, FP32 A-images; ms[6] lockstep iterations.  colcells: sum over
 * subdomain-iterations of (basis columns x cells), the unit of the Gram and update traffic. */
int pmf_get_eig_phases(pmf_solver* s, double ms[8], unsigned long long* colcells);

/* Launch-shape tuner table of this process as JSON ({"<kernel>|<shape>|<device>": {"choice": c,
 * "us": [per-candidate microseconds]}, ...}).  Copies at most len-1 bytes and a terminating zero into
 * buf (buf may be NULL); returns the full length.  The tuner is on unless PMF_AUTOTUNE=0 or
 * -pmf_autotune 0; PMF_TUNE_FILE=<path> keeps the table across processes. */
int pmf_tune_report(char* buf, int len);

/* total number of CUDA kernels launched by this library in this process */
unsigned long long pmf_launch_count(void);

const char* pmf_last_error(void);
int pmf_device_count(void);

#ifdef __cplusplus
}
#endif

#endif
