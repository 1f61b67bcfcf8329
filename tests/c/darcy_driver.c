/*
 * A driver program written only against PreMixFEM_3D.h, in the way the
 * reference's experiment drivers use it (PC_init -> kappa on the DM ->
 * PC_create_A -> KSPCG with the PCSHELL -> KSPSolve -> PC_print_stat ->
 * PC_final).  Compiled with plain gcc and linked against
 * libpremixfem_b200.so; the GPU tests run it and compare with the oracle.
 *
 * Problem: the periodic cross-channel permeability (k = 10^cr where the cell
 * index modulo 8 lies in [3, 5) along two of the three axes, else 1) with
 * the zero-sum well source (+1e3|K| at the four vertical corner columns,
 * -1e3|K| at the four centre columns), homogeneous Neumann boundary, on the
 * unit cube with size^3 cells; the right-hand side is normalised to unit
 * length before the solve.
 *
 * Options: -size n, -cr c, -petsc_default (plain CG, no preconditioner),
 * -out path (write the solution as raw little-endian doubles, x fastest),
 * plus every PC_init / KSP option.
 */
#include <math.h>
#include <stdio.h>

#include "PreMixFEM_3D.h"

static int in_band(PetscInt e) {
  const PetscInt r = e % 8;
  return r >= 3 && r < 5;
}

static PetscErrorCode build_kappa(PCCtx *ctx, PetscInt cr) {
  PetscInt x0, y0, z0, nx, ny, nz, ex, ey, ez, d;
  PetscScalar ***k[DIM];
  const PetscScalar hi = pow(10.0, (double)cr);
  PetscFunctionBeginUser;
  PetscCall(DMDAGetCorners(ctx->dm, &x0, &y0, &z0, &nx, &ny, &nz));
  for (d = 0; d < DIM; ++d) {
    PetscCall(DMCreateGlobalVector(ctx->dm, &ctx->kappa[d]));
    PetscCall(DMDAVecGetArray(ctx->dm, ctx->kappa[d], &k[d]));
  }
  for (ez = z0; ez < z0 + nz; ++ez)
    for (ey = y0; ey < y0 + ny; ++ey)
      for (ex = x0; ex < x0 + nx; ++ex) {
        const int ch = (in_band(ex) && in_band(ey)) || (in_band(ex) && in_band(ez)) || (in_band(ey) && in_band(ez));
        for (d = 0; d < DIM; ++d) k[d][ez][ey][ex] = ch ? hi : 1.0;
      }
  for (d = 0; d < DIM; ++d) PetscCall(DMDAVecRestoreArray(ctx->dm, ctx->kappa[d], &k[d]));
  PetscFunctionReturn(0);
}

static PetscErrorCode build_source(PCCtx *ctx, Vec *b) {
  PetscInt x0, y0, z0, nx, ny, nz, ex, ey, ez;
  PetscScalar ***s;
  const PetscScalar q = 1.0e3 * ctx->H_x * ctx->H_y * ctx->H_z;
  PetscFunctionBeginUser;
  PetscCall(DMCreateGlobalVector(ctx->dm, b));
  PetscCall(DMDAGetCorners(ctx->dm, &x0, &y0, &z0, &nx, &ny, &nz));
  PetscCall(DMDAVecGetArray(ctx->dm, *b, &s));
  for (ez = z0; ez < z0 + nz; ++ez)
    for (ey = y0; ey < y0 + ny; ++ey)
      for (ex = x0; ex < x0 + nx; ++ex) {
        const int corner = (ex == 0 || ex == ctx->M - 1) && (ey == 0 || ey == ctx->N - 1);
        const int centre = (ex == ctx->M / 2 - 1 || ex == ctx->M / 2) && (ey == ctx->N / 2 - 1 || ey == ctx->N / 2);
        s[ez][ey][ex] = corner ? q : (centre ? -q : 0.0);
      }
  PetscCall(DMDAVecRestoreArray(ctx->dm, *b, &s));
  PetscFunctionReturn(0);
}

int main(int argc, char **argv) {
  PetscInt mesh[3] = {16, 16, 16}, cr = 0, d, its = 0, n = 0;
  PetscScalar dom[3] = {1.0, 1.0, 1.0}, bnorm, res;
  PetscBool plain = PETSC_FALSE;
  const char *out = NULL;
  PCCtx ctx;
  Vec b, x, r;
  Mat A;
  KSP ksp;
  int i;

  PetscCall(SlepcInitialize(&argc, &argv, NULL, "cross-channel Darcy driver"));
  PetscCall(PetscOptionsGetInt(NULL, NULL, "-size", &mesh[0], NULL));
  mesh[1] = mesh[2] = mesh[0];
  PetscCall(PetscOptionsGetInt(NULL, NULL, "-cr", &cr, NULL));
  PetscCall(PetscOptionsHasName(NULL, NULL, "-petsc_default", &plain));
  for (i = 1; i + 1 < argc; ++i)
    if (strcmp(argv[i], "-out") == 0) out = argv[i + 1];

  PetscCall(PC_init(&ctx, dom, mesh));
  PetscCall(PC_print_info(&ctx));
  PetscCall(build_kappa(&ctx, cr));
  PetscCall(PC_create_A(&ctx, &A));
  PetscCall(build_source(&ctx, &b));
  PetscCall(VecNormalize(b, &bnorm));

  PetscCall(KSPCreate(PETSC_COMM_WORLD, &ksp));
  PetscCall(KSPSetOperators(ksp, A, A));
  if (!plain) {
    PC pc;
    PetscCall(KSPGetPC(ksp, &pc));
    PetscCall(PCSetType(pc, PCSHELL));
    PetscCall(PCShellSetContext(pc, &ctx));
    PetscCall(PCShellSetSetUp(pc, PC_setup));
    PetscCall(PCShellSetApply(pc, PC_apply_vec));
    PetscCall(PCShellSetName(pc, "three-level GMsFEM"));
  }
  PetscCall(KSPSetNormType(ksp, KSP_NORM_UNPRECONDITIONED));
  PetscCall(KSPSetFromOptions(ksp));
  PetscCall(KSPSetUp(ksp));
  PetscCall(VecDuplicate(b, &x));
  PetscCall(KSPSolve(ksp, b, x));

  PetscCall(VecDuplicate(x, &r));
  PetscCall(MatMult(A, x, r));
  PetscCall(VecAXPY(r, -1.0, b));
  PetscCall(VecNorm(r, NORM_2, &res));
  PetscCall(VecNorm(b, NORM_2, &bnorm));
  PetscCall(KSPGetIterationNumber(ksp, &its));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD, "iterations=%d\n", its));
  PetscCall(PetscPrintf(PETSC_COMM_WORLD, "residual=%.6e rhs=%.6e\n", res, bnorm));
  PetscCall(KSPConvergedReasonView(ksp, NULL));
  if (!plain) PetscCall(PC_print_stat(&ctx));

  if (out) {
    const PetscScalar *a;
    FILE *f = fopen(out, "wb");
    PetscCheck(f != NULL, PETSC_COMM_WORLD, PETSC_ERR_USER, "cannot open %s\n", out);
    PetscCall(VecGetSize(x, &n));
    PetscCall(VecGetArrayRead(x, &a));
    fwrite(a, sizeof(PetscScalar), (size_t)n, f);
    PetscCall(VecRestoreArrayRead(x, &a));
    fclose(f);
  }

  PetscCall(VecDestroy(&r));
  PetscCall(KSPDestroy(&ksp));
  PetscCall(VecDestroy(&x));
  PetscCall(VecDestroy(&b));
  for (d = 0; d < DIM; ++d) PetscCall(VecDestroy(&ctx.kappa[d]));
  PetscCall(MatDestroy(&A));
  if (!plain)
    PetscCall(PC_final(&ctx));
  else
    PetscCall(PC_final_default(&ctx));
  PetscCall(SlepcFinalize());
  return 0;
}
