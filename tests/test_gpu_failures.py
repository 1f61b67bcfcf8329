"""Failure paths of the solve on the GPU, each caused by a host-side input.

The reference stops with a PETSc error where its libraries fail:
  * SLEPc finds fewer than en_lv1 local eigenpairs (src/PreMixFEM_3D.c:367,
    PETSC_ERR_USER; level 3 at :1098) -- here with -pmf_eig_require_converged,
    since by default a local eigensolve that spends its iterations keeps its
    last Ritz block;
  * a factorisation meets a zero pivot (the local KSPs are set up with
    KSPSetErrorIfNotConverged, :212, :725, :903, :1376);
  * PETSc's KSPConvergedDefault ends a solve whose residual norm is NaN or Inf
    with KSP_DIVERGED_NANORINF.
The library returns the same PETSc error codes (83, 71) from pmf_setup and the
reason code 4 from pmf_solve, and the CUDA context stays usable: every test
solves a clean problem afterwards.  None of these inputs can fault the GPU:
NaN and Inf propagate through the arithmetic, and every loop they reach is
bounded by an iteration count.
"""
import numpy as np
import pytest

from premixfem_b200 import fields
from premixfem_b200._native import PmfError
from premixfem_b200.solver import DarcySolver, options_string

pytestmark = pytest.mark.gpu

OPTS = {"sd": 2, "en_lv1": 4, "en_lv2": 4}


def _clean_solve(precision="fp64"):
    prob = fields.unit_cube_grf(16, seed=1)
    s = DarcySolver.from_problem(prob, options_string(dict(OPTS, pmf_precision=precision)))
    s.setup()
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    s.close()
    assert reason == "converged" and its > 0
    return its


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_in_rhs_gives_diverged_nanorinf(native, precision):
    prob = fields.unit_cube_grf(16, seed=1)
    s = DarcySolver.from_problem(prob, options_string(dict(OPTS, pmf_precision=precision)))
    s.setup()
    b = s.rhs(prob["source"].ravel())
    bad = b.copy()
    bad[1234] = np.nan
    x, its, rnorm, reason = s.solve(bad)
    assert reason == "diverged_nanorinf"
    assert its == 0  # the initial residual norm is already NaN
    # the same solver object solves the clean right-hand side afterwards
    x, its, rnorm, reason = s.solve(b)
    assert reason == "converged" and its > 0
    inf_b = b.copy()
    inf_b[7] = np.inf
    _, its, _, reason = s.solve(inf_b)
    assert reason == "diverged_nanorinf" and its == 0
    s.close()


@pytest.mark.parametrize("bad_kappa", [0.0, -1.0])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonpositive_kappa_gives_zero_pivot_error(native, bad_kappa, precision):
    prob = fields.unit_cube_grf(16, seed=2)
    kx, ky, kz = (np.array(k, copy=True) for k in prob["kappa"])
    for k in (kx, ky, kz):
        k[3, 9, 5] = bad_kappa  # one cell
    s = DarcySolver(prob["dom"], prob["mesh"], options_string(dict(OPTS, pmf_precision=precision)))
    s.set_kappa(kx, ky, kz)
    for f, v in prob["dirichlet"].items():
        s.set_dirichlet(f, v)
    with pytest.raises(PmfError) as e:
        s.setup()
    assert e.value.code == 71, e.value
    assert "pivot" in str(e.value)
    s.close()
    _clean_solve(precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eigensolver_iteration_budget(native, precision):
    prob = fields.unit_cube_grf(16, seed=3)
    opts = options_string(dict(OPTS, pmf_precision=precision, pmf_eig_max_it=1))
    s = DarcySolver.from_problem(prob, opts + " -pmf_eig_require_converged")
    with pytest.raises(PmfError) as e:
        s.setup()
    assert e.value.code == 83, e.value
    assert "did not converge" in str(e.value)
    s.close()
    # by default the one-step Ritz blocks are kept: the set-up completes,
    # reports status 1 (max_it) and the solve still converges
    s = DarcySolver.from_problem(prob, opts)
    s.setup()
    ev, ks, iters, status = s.eigen_lv1()
    assert (status == 1).any()
    assert iters.max() <= 1
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    assert reason == "converged"
    assert rnorm <= 1e-8 * np.linalg.norm(b) * (1 + 1e-6)
    s.close()
    _clean_solve(precision)


def test_max_it_reason(native):
    prob = fields.unit_cube_grf(16, seed=1)
    s = DarcySolver.from_problem(prob, options_string(dict(OPTS, ksp_max_it=3)))
    s.setup()
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    s.close()
    assert reason == "diverged_its" and its == 3
