"""The C++/OpenMP CPU restatement (oracle/cpu_ref) against the NumPy oracle.

The restatement is the timed CPU baseline, so it has to compute the same
method: same partition, operator, local eigenspaces, coarse levels, cycle and
CG recurrence.  Its local eigensolver is LOBPCG instead of a dense solve, so
agreement is to the eigensolver tolerance, not bit for bit.
"""
import numpy as np
import pytest

from oracle import pmf_oracle as O
from oracle.cpu_ref import pmf_cpu as CR
from premixfem_b200 import fields


@pytest.fixture(scope="module", autouse=True)
def _built():
    CR.build()


def _aniso_box(mesh, seed, dirichlet):
    prob = fields.random_box(mesh, seed=seed, sigma=1.5, dirichlet=dirichlet)
    kx, ky, kz = prob["kappa"]
    rng = np.random.default_rng(seed + 100)
    return dict(prob, kappa=(kx, ky * 0.1, kz * np.exp(rng.standard_normal(kz.shape))))


CASES = [
    ("grf16_mod", lambda: fields.unit_cube_grf(16, seed=1), dict(sd=2, en_lv1=4, en_lv2=4, eg_op=0)),
    ("grf16_vranks_mean", lambda: fields.unit_cube_grf(16, seed=2),
     dict(sd=2, vranks=(2, 2, 1), en_lv1=4, en_lv2=4, eg_op=1)),
    ("grf16_wcycle_diag", lambda: fields.unit_cube_grf(16, seed=3),
     dict(sd=2, vranks=(2, 1, 1), en_lv1=3, en_lv2=3, eg_op=2, use_W_cycle=True, si_lv1=2, si_lv2=2)),
    ("ragged_aniso", lambda: _aniso_box((13, 11, 9), 7, {"y+": 0.5, "z-": -1.0}),
     dict(sd=(2, 2, 1), vranks=(2, 1, 2), en_lv1=3, en_lv2=2, eg_op=0)),
    ("grf16_2level", lambda: fields.unit_cube_grf(16, seed=2), dict(sd=2, vranks=(2, 2, 1), en_lv1=4, use_2level=True)),
    ("aniso_2level_si2", lambda: dict(fields.aniso_const(8, 8, 8), dirichlet={"z+": 1.0}),
     dict(sd=2, en_lv1=3, use_2level=True, si_lv1=2)),
    ("grf16_full_cholesky", lambda: fields.unit_cube_grf(16, seed=1),
     dict(sd=2, en_lv1=4, en_lv2=4, use_full_Cholesky_lv1=True)),
    ("ragged_full_cholesky", lambda: fields.random_box((13, 11, 9), seed=7, sigma=2.0),
     dict(sd=(2, 2, 1), vranks=(2, 1, 3), en_lv1=3, en_lv2=2, use_full_Cholesky_lv1=True)),
]


@pytest.mark.parametrize("name,make,opts", CASES, ids=[c[0] for c in CASES])
def test_matches_oracle(name, make, opts):
    prob = make()
    ref = O.solve(prob, O.Options(**opts))
    got = CR.solve(prob, **opts)
    assert got["eig_unconverged"] == 0
    assert abs(got["its"] - ref["its"]) <= 1, (got["its"], ref["its"])
    err = np.linalg.norm(got["x"] - ref["x"]) / np.linalg.norm(ref["x"])
    assert err < 1e-8, err
    assert got["rnorm"] <= 1e-8 * got["r0"]


def test_pure_neumann_solution():
    # no Dirichlet face: A is singular and the level-3 matrix gets the NIL shift, so
    # the constant component of the iterates is set by rounding (1 / NIL times a
    # residual mean near machine precision) and the iteration count is
    # rounding-sensitive; compare modulo constants.
    prob = fields.aniso_const(8, 8, 8)
    opts = dict(sd=2, en_lv1=4, en_lv2=4)
    ref = O.solve(prob, O.Options(**opts))
    got = CR.solve(prob, **opts)
    assert abs(got["its"] - ref["its"]) <= 3, (got["its"], ref["its"])
    a = ref["x"] - ref["x"].mean()
    b = got["x"] - got["x"].mean()
    err = np.linalg.norm(b - a) / np.linalg.norm(a)
    assert err < 1e-8, err


def test_pure_neumann_without_shift_matches_oracle():
    # -no_shift_A_cc: the null pivot of the level-3 matrix is dropped, so the
    # iteration count no longer depends on rounding and must match
    prob = fields.aniso_const(8, 8, 8)
    opts = dict(sd=2, en_lv1=4, en_lv2=4, no_shift_A_cc=True)
    ref = O.solve(prob, O.Options(**opts))
    got = CR.solve(prob, **opts)
    assert got["its"] == ref["its"]
    a, b = ref["x"] - ref["x"].mean(), got["x"] - got["x"].mean()
    assert np.linalg.norm(b - a) <= 1e-8 * np.linalg.norm(a)


def test_adaptive_eigenvector_counts_match_oracle():
    # -eb_lv1 / -eb_lv2 (:369-383, :1100-1115) halfway between neighbouring order
    # statistics of the oracle's eigenvalues, so that the counts vary across
    # subdomains and ranks and no eigenvalue sits on a threshold
    prob = fields.unit_cube_grf(16, seed=5)
    base = dict(sd=2, vranks=(2, 2, 1), en_lv1=6, en_lv2=4)
    pc = O.solve(prob, O.Options(**base))["pc"]
    w3 = np.sort([w[3] for w in pc.eigvals_lv1])
    v1 = np.sort([w[1] for w in pc.eigvals_lv2])
    h = len(w3) // 2
    opts = dict(base, eb_lv1=0.5 * (w3[h - 1] + w3[h]), eb_lv2=0.5 * (v1[1] + v1[2]))
    ref = O.solve(prob, O.Options(**opts))
    counts1, counts2 = ref["pc"].eig_num_lv1, ref["pc"].eig_num_lv2
    assert min(counts1) < max(counts1) and min(counts2) < 4
    got = CR.solve(prob, **opts)
    assert got["n3"] == sum(counts2)
    assert abs(got["its"] - ref["its"]) <= 1, (got["its"], ref["its"])
    assert np.linalg.norm(got["x"] - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])


def test_large_coarse_level_uses_the_smallest_eigenpairs_only():
    # 256 subdomains of 4 x 4 x 8 cells, k = 4: 1 024 coarse unknowns on one rank,
    # so the restatement's level-3 HEP takes the inverse subspace iteration for its
    # 4 smallest eigenpairs instead of a full dense eigendecomposition
    prob = fields.unit_cube_grf(32, seed=6)
    opts = dict(sd=(8, 8, 4), en_lv1=4, en_lv2=4)
    ref = O.solve(prob, O.Options(**opts))
    got = CR.solve(prob, **opts)
    assert got["n3"] == 4
    assert abs(got["its"] - ref["its"]) <= 1, (got["its"], ref["its"])
    assert np.linalg.norm(got["x"] - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])


def test_rejects_too_many_eigenvectors():
    prob = fields.random_box((4, 4, 4), seed=1)
    with pytest.raises(ValueError):
        CR.solve(prob, sd=2, en_lv1=9)  # 2^3-cell subdomains cannot hold 9 vectors


def test_thread_count_does_not_change_the_result():
    prob = fields.unit_cube_grf(16, seed=4)
    a = CR.solve(prob, sd=2, threads=1)
    b = CR.solve(prob, sd=2, threads=4)
    assert a["its"] == b["its"]
    assert np.linalg.norm(a["x"] - b["x"]) <= 1e-10 * np.linalg.norm(a["x"])


# Reduced copies of the other benchmark distributions.  The layered channel
# field keeps the 10 x 10 x 5 subdomains, 20 x 10 x 2 cells and 1e6 channel
# contrast of the 60 x 220 x 85 workload; the large fracture field keeps
# sigma 3 and the 1e6 fracture planes of the 512 x 512 x 256 one, with k = 8
# eigenvectors.


def test_layered_channels_match_oracle():
    # Pure Neumann with a zero-sum injector/producer pair.  Without a null space
    # the CG recurrence stalls on the constant direction before 1e-8 (PETSc's
    # DIVERGED_INDEFINITE); with -ksp_constant_null_space both solves converge
    # to the direct solution.
    prob = fields.layered(seed=2, M=20, N=30, P=10, smooth_layers=4)
    opts = dict(sd=(2, 3, 2), en_lv1=4, en_lv2=4)
    plain = O.solve(prob, O.Options(**opts))
    assert plain["reason"] == "diverged_indefinite"
    ref = O.solve(prob, O.Options(**opts, constant_null_space=True))
    assert ref["reason"] == "converged_rtol"
    xd = O.direct_solve(ref["op"], ref["b"])
    a = ref["x"] - ref["x"].mean()
    assert np.linalg.norm(a - (xd - xd.mean())) <= 1e-8 * np.linalg.norm(xd - xd.mean())
    got = CR.solve(prob, **opts, constant_null_space=True)
    assert got["eig_unconverged"] == 0
    assert got["rnorm"] <= 1e-8 * got["r0"]
    assert abs(got["its"] - ref["its"]) <= 1, (got["its"], ref["its"])
    b = got["x"] - got["x"].mean()
    err = np.linalg.norm(b - a) / np.linalg.norm(a)
    assert err < 1e-8, err



def test_large_fracture_field_matches_oracle():
    prob = fields.large_frac(M=32, N=32, P=16, seed=5, n_frac=8, frac_lo=4, frac_hi=32)
    opts = dict(sd=(4, 4, 2), en_lv1=8, en_lv2=4)
    ref = O.solve(prob, O.Options(**opts))
    got = CR.solve(prob, **opts)
    assert got["eig_unconverged"] == 0
    assert abs(got["its"] - ref["its"]) <= 1, (got["its"], ref["its"])
    err = np.linalg.norm(got["x"] - ref["x"]) / np.linalg.norm(ref["x"])
    assert err < 1e-8, err


def test_problem_batch_every_rhs_matches_oracle():
    # independent ragged problems of the batching workload, four right-hand
    # sides each through one preconditioner set-up of the oracle
    # (one set-up and four right-hand sides in the restatement too)
    for prob, sources in fields.grf_batch(count=3, seed=3, lo=10, hi=20):
        opts = dict(sd=fields.tiles(prob["mesh"]), en_lv1=4, en_lv2=4)
        op = O.Operator(prob)
        pc = O.Preconditioner(op, O.Options(**opts))
        got = CR.solve(prob, sources=sources, **opts)
        its_ref = []
        for q, src in enumerate(sources):
            b = O.Operator(dict(prob, source=src)).rhs()
            x_ref, its, _, reason = O.pcg(op.A, b, pc.apply)
            assert reason == "converged_rtol"
            its_ref.append(its)
            err = np.linalg.norm(got["x"][q] - x_ref) / np.linalg.norm(x_ref)
            assert err < 1e-8, (prob["mesh"], q, err)
        assert abs(got["its"] - its_ref[0]) <= 1, (prob["mesh"], got["its"], its_ref)
        assert abs(got["its_max"] - max(its_ref)) <= 1, (prob["mesh"], got["its_max"], its_ref)


def test_eigenvalue_relative_stopping_rule_on_channels():
    # The local eigensolves stop at ||r_j||_{M^-1} <= tol x lscale (lscale = max
    # diag(A_N) / M).  On channel fields the smallest eigenvalues lie far below
    # lscale, the coarse space they give is too loose, and CG stalls above 1e-8.
    # -pmf_eig_rel_floor 1e-4 tests against max(|lambda_j|, 1e-4 lscale) instead
    # and reaches the dense-eigensolver oracle's iteration count and solution.
    prob = fields.layered(seed=2, M=20, N=20, P=10, smooth_layers=4, contrast=1e4)
    opts = dict(sd=(2, 2, 2), en_lv1=4, en_lv2=4)
    ref = O.solve(prob, O.Options(**opts, constant_null_space=True))
    assert ref["reason"] == "converged_rtol"
    loose = CR.solve(prob, **opts, constant_null_space=True, max_it=300)
    assert loose["rnorm"] > 1e-8 * loose["r0"]
    got = CR.solve(prob, **opts, constant_null_space=True, eig_rel_floor=1e-4)
    assert got["rnorm"] <= 1e-8 * got["r0"]
    assert abs(got["its"] - ref["its"]) <= 1, (got["its"], ref["its"])
    a = ref["x"] - ref["x"].mean()
    err = np.linalg.norm(got["x"] - got["x"].mean() - a) / np.linalg.norm(a)
    assert err < 1e-8, err
