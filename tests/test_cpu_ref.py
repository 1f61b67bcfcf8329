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
