"""GPU parity: libpremixfem_b200.so (through the C ABI) against the CPU oracle.

Tolerances (FP64 plain form unless stated):
  * operator A x and the right-hand side: 1e-13 relative (same arithmetic);
  * local (level-2) and level-3 eigenvalues: 1e-6 relative, with an absolute
    floor of 1e-9 x the largest wanted eigenvalue for the zero (constant) modes;
  * one preconditioner application: 1e-6 relative L2 (the eigenvectors are
    converged to a 1e-6 residual, not to machine precision);
  * PCG: iteration count within +-1 of the oracle, solution within 1e-8
    relative L2 of an FP64 direct solve;
  * mixed precision (FP32 preconditioner, FP64 PCG): iterations within +-1 of
    the oracle, same 1e-8 solution bound.
"""
import os

import numpy as np
import pytest

from oracle import pmf_oracle as O
from premixfem_b200 import fields
from premixfem_b200.solver import DarcySolver, options_string

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle_opts(d):
    o = O.Options()
    for k, v in d.items():
        if k == "pmf_vranks":
            o.vranks = tuple(v)
        elif k == "pmf_sd":
            o.sd = tuple(v)
        elif k == "pmf_precision":
            continue
        else:
            setattr(o, k, v)
    return o


def _gpu(problem, d):
    s = DarcySolver.from_problem(problem, options_string(d))
    s.setup()
    return s


CASES = {
    "grf16_sd2": (lambda: fields.unit_cube_grf(16, seed=1), {"sd": 2, "en_lv1": 4, "en_lv2": 4}),
    "grf16_vr222": (lambda: fields.unit_cube_grf(16, seed=3),
                    {"sd": 2, "pmf_vranks": (2, 2, 2), "en_lv1": 4, "en_lv2": 3}),
    "ragged_vr": (lambda: fields.random_box((13, 11, 9), seed=7, sigma=2.0),
                  {"pmf_sd": (2, 2, 1), "pmf_vranks": (2, 1, 3), "en_lv1": 3, "en_lv2": 2}),
    "cross16_cr3": (lambda: dict(fields.cross(16, 3), dirichlet={"x-": 0.0}),
                    {"sd": 2, "pmf_vranks": (1, 2, 2), "en_lv1": 4, "en_lv2": 4}),
    "aniso_wcycle": (lambda: dict(fields.aniso_const(8, 8, 8), dirichlet={"z+": 1.0}),
                     {"sd": 2, "en_lv1": 3, "en_lv2": 2, "use_W_cycle": True}),
    # one virtual rank of 144 subdomains: 576 coarse unknowns, past the cluster
    # inverse (384), so the rank's level-2 and rank-Neumann inverses take the
    # panel Gauss-Jordan over nine 64-pivot panels
    "grf24_rank576": (lambda: fields.unit_cube_grf(24, seed=5), {"pmf_sd": (6, 6, 4), "en_lv1": 4, "en_lv2": 4}),
    # 1 000 subdomains in one rank, 2 000 coarse unknowns: the level-3 eigensolver's
    # block no longer fits in shared memory and runs as multi-CTA phases
    "grf40_rank2000": (lambda: fields.unit_cube_grf(40, seed=6), {"pmf_sd": (10, 10, 10), "en_lv1": 2, "en_lv2": 4}),
}


@pytest.fixture(scope="module")
def oracle_cache():
    return {}


def _oracle(name, cache):
    if name not in cache:
        mk, d = CASES[name]
        prob = mk()
        cache[name] = (prob, d, O.solve(prob, _oracle_opts(d)))
    return cache[name]


def test_operator_and_rhs(native):
    prob = fields.random_box((11, 7, 5), seed=2, sigma=2.0, dirichlet={"x-": 1.0, "y+": 0.5})
    op = O.Operator(prob)
    s = DarcySolver.from_problem(prob, "-sd 2")
    s.setup()
    x = np.random.default_rng(0).standard_normal(op.n)
    y = s.apply_A(x)
    ref = op.A @ x
    assert np.linalg.norm(y - ref) <= 1e-13 * np.linalg.norm(ref)
    b = s.rhs(prob["source"].ravel())
    np.testing.assert_allclose(b, op.rhs(), rtol=1e-14, atol=1e-14 * np.abs(op.rhs()).max())
    s.close()


@pytest.mark.parametrize("name", list(CASES))
def test_local_and_level3_eigenvalues(native, name, oracle_cache):
    prob, d, ref = _oracle(name, oracle_cache)
    s = _gpu(prob, d)
    ev, ks, iters, status = s.eigen_lv1()
    pc = ref["pc"]
    # status 0: converged to tolerance, 2: stopped at the rounding floor within 100 x tol, 1: max_it
    assert (status != 1).all(), f"LOBPCG did not converge on {np.nonzero(status == 1)[0]}"
    ref1 = np.stack(pc.eigvals_lv1)
    scale = np.abs(ref1).max(axis=1, keepdims=True)
    err = np.abs(ev - ref1) / np.maximum(np.abs(ref1), 1e-3 * scale)
    assert err.max() <= 1e-6, f"max rel eigen error {err.max():.2e}"
    ev3, ks3, _ = s.eigen_lv2()
    ref3 = np.stack([w for w in pc.eigvals_lv2])
    scale3 = np.abs(ref3).max(axis=1, keepdims=True)
    err3 = np.abs(ev3 - ref3) / np.maximum(np.abs(ref3), 1e-3 * scale3)
    assert err3.max() <= 1e-6, f"max rel level-3 eigen error {err3.max():.2e}"
    s.close()


@pytest.mark.parametrize("name", list(CASES))
def test_pc_apply_matches_oracle(native, name, oracle_cache):
    prob, d, ref = _oracle(name, oracle_cache)
    s = _gpu(prob, d)
    x = np.random.default_rng(11).standard_normal(ref["op"].n)
    y = s.pc_apply(x)
    yr = ref["pc"].apply(x)
    rel = np.linalg.norm(y - yr) / np.linalg.norm(yr)
    assert rel <= 1e-6, f"PC_apply_vec relative difference {rel:.2e}"
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_pcg_iterations_and_solution(native, name, precision, oracle_cache):
    prob, d, ref = _oracle(name, oracle_cache)
    s = _gpu(prob, dict(d, pmf_precision=precision))
    op = ref["op"]
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    assert reason == "converged"
    assert abs(its - ref["its"]) <= 1, f"iterations {its} vs oracle {ref['its']}"
    assert np.linalg.norm(b - op.A @ x) <= 1e-8 * np.linalg.norm(b) * (1 + 1e-6)
    xd = O.direct_solve(op, ref["b"])
    if not op.dir_faces:
        x = x - x.mean()
        xd = xd - xd.mean()
    err = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    assert err <= 1e-8, f"solution error vs direct {err:.2e}"
    s.close()


def test_device_pointer_path_matches_host_path(native):
    torch = pytest.importorskip("torch")
    prob = fields.unit_cube_grf(16, seed=5)
    s = DarcySolver.from_problem(prob, "-sd 2")
    s.setup()
    b = s.rhs(prob["source"].ravel())
    xh, its_h, _, _ = s.solve(b)
    bd = torch.from_numpy(b).cuda()
    xd, its_d, _, _ = s.solve(bd)
    assert its_h == its_d
    np.testing.assert_array_equal(xd.cpu().numpy(), xh)
    s.close()


def test_bad_arguments_return_errors(native):
    from premixfem_b200._native import PmfError
    with pytest.raises(PmfError) as e:
        DarcySolver((1, 1, 1), (0, 4, 4), "")
    assert e.value.code == 62
    with pytest.raises(PmfError) as e:
        DarcySolver((1, 1, 1), (8, 8, 8), "-eg_op 7")
    assert e.value.code == 62
    s = DarcySolver((1, 1, 1), (8, 8, 8), "-sd 2")
    with pytest.raises(PmfError) as e:
        s.setup()  # kappa not set
    assert e.value.code == 73
    s.close()


TWO_LEVEL = {
    "grf16_2level": (lambda: fields.unit_cube_grf(16, seed=2),
                     {"sd": 2, "pmf_vranks": (2, 2, 1), "en_lv1": 4, "use_2level": True}),
    "aniso_2level_si2": (lambda: dict(fields.aniso_const(8, 8, 8), dirichlet={"z+": 1.0}),
                         {"sd": 2, "en_lv1": 3, "use_2level": True, "si_lv1": 2}),
    # 13^3 subdomains of 4^3 cells, 8 788 coarse unknowns: above the dense
    # coarse solver's former 8 192 limit, through the banded Cholesky
    "grf52_2level_banded": (lambda: fields.unit_cube_grf(52, seed=4),
                            {"sd": 13, "en_lv1": 4, "use_2level": True}),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(TWO_LEVEL))
def test_two_level_matches_oracle(native, name, precision, oracle_cache):
    """-use_2level (_PC_setup_lv2_c / _PC_apply_vec_lv2_2level): one preconditioner
    application (FP64 only, 1e-6) and the PCG iterations (+-1) and solution (1e-8)."""
    mk, d = TWO_LEVEL[name]
    key = ("two_level", name)
    if key not in oracle_cache:
        p_ = mk()
        oracle_cache[key] = (p_, O.solve(p_, _oracle_opts(d)))
    prob, ref = oracle_cache[key]
    s = _gpu(prob, dict(d, pmf_precision=precision))
    if precision == "fp64":
        x = np.random.default_rng(12).standard_normal(ref["op"].n)
        y, yr = s.pc_apply(x), ref["pc"].apply(x)
        assert np.linalg.norm(y - yr) <= 1e-6 * np.linalg.norm(yr)
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    assert reason == "converged"
    assert abs(its - ref["its"]) <= 1, f"iterations {its} vs oracle {ref['its']}"
    xd = O.direct_solve(ref["op"], ref["b"])
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    s.close()


CHOL_CASES = {
    "grf16_chol": (lambda: fields.unit_cube_grf(16, seed=1),
                   {"sd": 2, "en_lv1": 4, "en_lv2": 4, "use_full_Cholesky_lv1": True}),
    "ragged_vr_chol": (lambda: fields.random_box((13, 11, 9), seed=7, sigma=2.0),
                       {"pmf_sd": (2, 2, 1), "pmf_vranks": (2, 1, 3), "en_lv1": 3, "en_lv2": 2,
                        "use_full_Cholesky_lv1": True}),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CHOL_CASES))
def test_full_cholesky_level1_matches_oracle(native, name, precision):
    """-use_full_Cholesky_lv1: exact banded Cholesky local solves against the
    oracle's exact local Cholesky (preconditioner output in FP64, PCG
    iterations +-1 and the solution within 1e-8 of a direct solve in both
    precisions)."""
    mk, d = CHOL_CASES[name]
    prob = mk()
    ref = O.solve(prob, _oracle_opts(d))
    s = _gpu(prob, dict(d, pmf_precision=precision))
    if precision == "fp64":
        x = np.random.default_rng(11).standard_normal(ref["op"].n)
        yr = ref["pc"].apply(x)
        rel = np.linalg.norm(s.pc_apply(x) - yr) / np.linalg.norm(yr)
        assert rel <= 1e-6, f"PC_apply_vec relative difference {rel:.2e}"
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    assert reason == "converged"
    assert abs(its - ref["its"]) <= 1, f"iterations {its} vs oracle {ref['its']}"
    xd = O.direct_solve(ref["op"], ref["b"])
    err = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    assert err <= 1e-8, f"solution error vs direct {err:.2e}"
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_final_phase_matches_persistent(native, precision):
    """The eigensolver's final Rayleigh-Ritz and output as phase kernels
    (-pmf_eig_final 1, the default) against the persistent mode-2 launch: the
    same local eigenvalues (1e-9 relative), preconditioner (1e-9 FP64, 1e-5
    mixed) and PCG iteration count (+-1)."""
    prob = fields.random_box((32, 24, 20), seed=4, sigma=1.5, dirichlet={"x-": 1.0})
    out = []
    for fin in (0, 1):
        s = _gpu(prob, {"pmf_sd": (4, 3, 2), "en_lv1": 5, "en_lv2": 3, "pmf_precision": precision, "pmf_eig_final": fin})
        ev = s.eigen_lv1()[0].copy()
        x = np.random.default_rng(2).standard_normal(32 * 24 * 20)
        y = s.pc_apply(x)
        b = s.rhs(prob["source"].ravel())
        _, its, _, reason = s.solve(b)
        assert reason == "converged"
        out.append((ev, y, its))
        s.close()
    ev0, ev1 = out[0][0], out[1][0]
    rel = np.abs(ev1 - ev0) / np.maximum(np.abs(ev0), 1e-9 * np.abs(ev0).max())
    assert rel.max() <= 1e-9, rel.max()
    tol = 1e-9 if precision == "fp64" else 1e-5
    ry = np.linalg.norm(out[1][1] - out[0][1]) / np.linalg.norm(out[0][1])
    assert ry <= tol, ry
    assert abs(out[1][2] - out[0][2]) <= 1


INIT_CASES = {
    # ragged 8 x 8 x 10 subdomains, one Dirichlet face (mass EIG_OP_MOD with the boundary term)
    "ragged_fp64": (lambda: fields.random_box((32, 24, 20), seed=4, sigma=1.5, dirichlet={"x-": 1.0}),
                    {"pmf_sd": (4, 3, 2), "en_lv1": 5, "en_lv2": 3, "pmf_precision": "fp64"}),
    "ragged_mixed": (lambda: fields.random_box((32, 24, 20), seed=4, sigma=1.5, dirichlet={"x-": 1.0}),
                     {"pmf_sd": (4, 3, 2), "en_lv1": 5, "en_lv2": 3, "pmf_precision": "mixed"}),
    # learned start from the shipped weights, then the random restart of the subdomains it leaves
    "fracture64_learned": (lambda: fields.fracture256(64, seed=3),
                           {"sd": 4, "en_lv1": 6, "en_lv2": 4, "pmf_precision": "mixed",
                            "pmf_learned": os.path.join(ROOT, "premixfem_b200", "weights", "fracture16_k6.pmfnet")}),
}


@pytest.mark.parametrize("case", sorted(INIT_CASES))
def test_batched_setup_phase_matches_persistent(native, case):
    """The eigensolver's set-up (mass and Neumann diagonals, IC(0) pivots, the
    initial block and its first Rayleigh-Ritz) as phase kernels
    (-pmf_eig_init 1) against the persistent mode-1 launch (the default):
    only the summation order of the first Grams differs, so in FP64 the local
    eigenvalues agree to 1e-6 relative with the floor of 1e-9 x the
    subdomain's largest wanted eigenvalue for the zero (constant) modes, and
    the PCG iteration count to +-1.  Mixed precision stores the basis in
    FP32: where that rounding flips in the first rotation, the two runs stop
    at different iterates of the 1e-6 residual test (||r||_{M^-1} <= 1e-6 x
    the largest diagonal-to-mass ratio, or 10 x that for a subdomain accepted
    at its rounding floor), and the eigenvalues agree to 5e-5 relative with
    a floor of 0.1 x the largest wanted one (the learned start, which runs to
    the same tolerance from the network's block, showed 1.6e-5)."""
    make, opts = INIT_CASES[case]
    prob = make()
    out = []
    for ini in (0, 1):
        s = _gpu(prob, dict(opts, pmf_eig_init=ini))
        ev = s.eigen_lv1()[0].copy()
        b = s.rhs(prob["source"].ravel())
        _, its, _, reason = s.solve(b)
        assert reason == "converged"
        out.append((ev, its))
        s.close()
    ev0, ev1 = out[0][0], out[1][0]
    scale = np.abs(ev0).max(axis=1, keepdims=True)
    rtol, floor = (5e-5, 1e-1) if opts["pmf_precision"] == "mixed" else (1e-6, 1e-3)
    rel = np.abs(ev1 - ev0) / np.maximum(np.abs(ev0), floor * scale)
    w = np.unravel_index(np.argmax(rel), rel.shape)
    assert rel.max() <= rtol, (rel.max(), w, ev0[w], ev1[w], scale[w[0], 0])
    assert abs(out[1][1] - out[0][1]) <= 1, (out[0][1], out[1][1])
