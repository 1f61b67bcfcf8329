/*
 * PreMixFEM_3D.h -- drop-in replacement of the reference's public header
 * (src/PreMixFEM_3D.h of Laphet/PreMixFEM) for the B200 library.
 *
 * Every entry point keeps the reference signature; the PETSc/MPI types come
 * from pmf_petsc_compat.h instead of petscksp.h/mpi.h.  Which reference
 * interface each declaration replaces:
 *   PCCtx            src/PreMixFEM_3D.h:32-45 (same field order and types)
 *   PC_init          src/PreMixFEM_3D.h:47  -> src/PreMixFEM_3D.c:1650-1741
 *   PC_print_info    src/PreMixFEM_3D.h:53  -> src/PreMixFEM_3D.c:1743-1755
 *   PC_setup         src/PreMixFEM_3D.h:55  -> src/PreMixFEM_3D.c:1826-1838 (PCSHELL set-up)
 *   PC_create_A      src/PreMixFEM_3D.h:57  -> src/PreMixFEM_3D.c:1757-1824
 *   PC_apply_vec     src/PreMixFEM_3D.h:59  -> src/PreMixFEM_3D.c:1840-1936 (PCSHELL apply)
 *   PC_get_range     src/PreMixFEM_3D.h:61  -> src/PreMixFEM_3D.c:1938-1952
 *   PC_print_stat    src/PreMixFEM_3D.h:63  -> src/PreMixFEM_3D.c:1954-1999
 *   PC_final_default src/PreMixFEM_3D.h:65  -> src/PreMixFEM_3D.c:2028-2046
 *   PC_final         src/PreMixFEM_3D.h:67  -> src/PreMixFEM_3D.c:2001-2026
 *   _PC_setup        src/PreMixFEM_3D.c:1392-1427 (called directly by src/test.c:85)
 *   mkl_serv_intel_cpu_true  src/PreMixFEM_3D.c:11-13 (kept as a no-op returning 1)
 *
 * Behaviour: PC_init reads the same options (-sd, -en_lv1, -en_lv2, -eb_lv1,
 * -eb_lv2, -si_lv1, -si_lv2, -eg_op, -use_W_cycle, -no_shift_A_cc; plus the
 * B200 extensions -pmf_sd a,b,c, -pmf_vranks px,py,pz and -pmf_precision
 * fp64|mixed) and creates s_ctx->dm; the caller builds s_ctx->kappa[0..2] on
 * that DM, exactly as with the reference.  The operator is the reference's
 * homogeneous-Neumann one (Dirichlet faces are offered by the flat ABI in
 * pmf_b200.h).  PC_create_A, PC_setup and PC_apply_vec run on the GPU.
 * KSPSolve of a KSPCG whose PCSHELL apply is PC_apply_vec, with
 * KSP_NORM_UNPRECONDITIONED as the reference drivers set, runs the whole
 * preconditioned CG on the device; any other PC or norm type runs PETSc's CG
 * recurrence on the host over the same callbacks.
 *
 * Differences a caller can see: -use_full_Cholesky_lv1 factors every
 * subdomain block as a banded Cholesky in natural order (bandwidth nx*ny, at
 * most 1800; the factors take cells * (nx*ny + 1) values of device memory), and
 * -use_2level needs a global coarse problem of at most 8192 unknowns (it is
 * solved densely); the multiscale bases stay in device memory, so
 * s_ctx->ms_bases_c / ms_bases_cc / ksp_lv1 hold NULL handles (the flat ABI's
 * pmf_get_phi reads the bases); the per-subdomain arrays (eigen_num_lv1, ...)
 * cover every subdomain of every virtual rank, and coarse_start/len* list the
 * subdomain slabs of the whole mesh along each axis.
 */
#ifndef YCQ_MIXFEM_3L3D_H
#define YCQ_MIXFEM_3L3D_H

#include "pmf_petsc_compat.h"

#define DIM 3
#define NEIGH 6
#define LEFT 1
#define RIGHT 2
#define DOWN 3
#define UP 4
#define BACK 5
#define FRONT 6
#define NIL 1.0e-12
#define MAX_LOG_STATES 10
#define STAGE_SU_LV1 0
#define STAGE_SU_LV2_1 1
#define STAGE_SU_LV2_2 2
#define STAGE_SU_LV3_1 3
#define STAGE_SU_LV3_2 4
#define STAGE_AV_LV1 5
#define STAGE_AV_LV2 6
#define STAGE_AV_LV3 7
#define STAGE_SU 8
#define STAGE_AV 9

#define EIG_OP_MOD 0
#define EIG_OP_MEAN 1
#define EIG_OP_DIAG 2

#ifdef __cplusplus
extern "C" {
#endif

typedef struct preconditioner_context {
  DM dm;
  Vec kappa[DIM], *ms_bases_c, *ms_bases_cc;
  KSP *ksp_lv1, ksp_lv2, ksp_lv3;
  PetscInt *coarse_startx, *coarse_lenx, *coarse_starty, *coarse_leny, *coarse_startz, *coarse_lenz;
  PetscInt smoothing_iters_lv1, smoothing_iters_lv2, sub_domains, lv2_eigen_op;
  PetscInt max_eigen_num_lv1, *eigen_num_lv1;
  PetscInt max_eigen_num_lv2, eigen_num_lv2;
  PetscScalar H_x, H_y, H_z, L, W, H;
  PetscScalar *eigen_max_lv1, *eigen_min_lv1, eigen_bd_lv1, eigen_max_lv2, eigen_min_lv2, eigen_bd_lv2;
  PetscScalar t_stages[MAX_LOG_STATES];
  PetscBool use_W_cycle, no_shift_A_cc, use_full_Cholesky_lv1, use_2level;
  PetscInt M, N, P;
} PCCtx;

PetscErrorCode PC_init(PCCtx *s_ctx, PetscScalar *dom, PetscInt *mesh);
/*
    dom[0], the length; dom[1], the width; dom[2], the height.
    mesh[0], partitions in x-direction; mesh[1], partitions in y-direction; mesh[2], partitions in z-direction.
*/

PetscErrorCode PC_print_info(PCCtx *s_ctx);

PetscErrorCode PC_setup(PC pc);

PetscErrorCode PC_create_A(PCCtx *s_ctx, Mat *A);

PetscErrorCode PC_apply_vec(PC pc, Vec x, Vec y);

PetscErrorCode PC_get_range(const void *sendbuff, void *recvbuff, MPI_Datatype datatype);

PetscErrorCode PC_print_stat(PCCtx *s_ctx);

PetscErrorCode PC_final_default(PCCtx *s_ctx);

PetscErrorCode PC_final(PCCtx *s_ctx);

PetscErrorCode _PC_setup(PCCtx *s_ctx);

int mkl_serv_intel_cpu_true();

#ifdef __cplusplus
}
#endif

#endif
