"""Reduced copies of the benchmark workloads on the GPU against the oracle.

  * layered channel field (the 60 x 220 x 85 workload's 10 x 10 x 5
    subdomains of 20 x 10 x 2 cells and 1e6 contrast, pure Neumann, with
    -ksp_constant_null_space) at 30 x 40 x 20;
  * the 512 x 512 x 256 workload's distribution (sigma 3 GRF, 1e6 fracture
    planes, p = 0 on z = 0, k = 8) at 32 x 32 x 16;
  * the 256^3 fracture workload's distribution at 128^3 with the shipped
    network weights and the default learned-start gate: sampled local
    eigenvalues against the oracle's exact local GHEPs, and the solution
    against the FP64 form solved to 1e-13.

Bars as in tests/test_gpu_parity.py: PCG iterations within +-1 of the oracle,
solutions within 1e-8 relative of an FP64 direct solve (compared modulo
constants for the pure-Neumann field), local eigenvalues within 1e-6 relative
(near-zero modes: 1e-9 of the subdomain's largest wanted eigenvalue).
"""
import os

import numpy as np
import pytest

from oracle import pmf_oracle as O
from premixfem_b200 import fields
from premixfem_b200.solver import DarcySolver, options_string

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "premixfem_b200", "weights", "fracture16_k6.pmfnet")


@pytest.fixture(scope="module")
def layered_ref():
    prob = fields.layered(seed=2, M=30, N=40, P=20, smooth_layers=8)
    opts = dict(sd=(3, 4, 4), en_lv1=4, en_lv2=4)
    ref = O.solve(prob, O.Options(**opts, constant_null_space=True))
    xd = O.direct_solve(ref["op"], ref["b"])
    return prob, opts, ref, xd - xd.mean()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_layered_channels_match_oracle(native, layered_ref, precision):
    prob, opts, ref, xd = layered_ref
    assert ref["reason"] == "converged_rtol"
    d = {"pmf_sd": opts["sd"], "en_lv1": 4, "en_lv2": 4, "pmf_precision": precision,
         "ksp_constant_null_space": True}
    s = DarcySolver.from_problem(prob, options_string(d))
    s.setup()
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    s.close()
    assert reason == "converged"
    assert abs(its - ref["its"]) <= 1, (its, ref["its"])
    err = np.linalg.norm((x - x.mean()) - xd) / np.linalg.norm(xd)
    assert err <= 1e-8, err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_fracture_field_matches_oracle(native, precision):
    prob = fields.large_frac(M=32, N=32, P=16, seed=5, n_frac=8, frac_lo=4, frac_hi=32)
    opts = dict(sd=(4, 4, 2), en_lv1=8, en_lv2=4)
    ref = O.solve(prob, O.Options(**opts))
    d = {"pmf_sd": opts["sd"], "en_lv1": 8, "en_lv2": 4, "pmf_precision": precision}
    s = DarcySolver.from_problem(prob, options_string(d))
    s.setup()
    ev, ks, iters, status = s.eigen_lv1()
    assert (status != 1).all()
    rel, null = O.eigenvalue_errors(ev, np.stack(ref["pc"].eigvals_lv1))
    assert rel <= 1e-6 and null <= 1e-9, (rel, null)
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    s.close()
    assert reason == "converged"
    assert abs(its - ref["its"]) <= 1, (its, ref["its"])
    xd = O.direct_solve(ref["op"], ref["b"])
    err = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    assert err <= 1e-8, err


def test_learned_start_accuracy_fracture128(native):
    """The learned start with the default gate on a field the network was not
    trained on: sampled local eigenvalues of the learned-start subdomains
    within the eigenvalue bar of the oracle, PCG iterations within +-1 of the
    FP64 form, and the solution's distance to the FP64 reference solution."""
    prob = fields.fracture256(128, seed=77)
    base = {"sd": 4, "pmf_vranks": (2, 2, 2), "en_lv1": 6, "en_lv2": 4}
    out = {}
    for form, extra in (("fp64_ref", {"pmf_precision": "fp64", "ksp_rtol": "1e-13"}),
                        ("fp64", {"pmf_precision": "fp64"}),
                        ("learned", {"pmf_precision": "mixed", "pmf_learned": WEIGHTS})):
        s = DarcySolver.from_problem(prob, options_string(dict(base, **extra)))
        s.setup()
        b = s.rhs(prob["source"].ravel())
        x, its, rnorm, reason = s.solve(b)
        ev, ks, iters, status = s.eigen_lv1()
        boxes = s.subdomains()[0]
        st = s.learned_stats() if form == "learned" else None
        s.close()
        assert reason == "converged", (form, reason)
        out[form] = dict(x=x, its=its, ev=ev, status=status, st=st)
    lr = out["learned"]
    assert lr["st"]["used"] == 1
    assert abs(lr["its"] - out["fp64"]["its"]) <= 1, (lr["its"], out["fp64"]["its"])
    assert (lr["status"] != 1).all()
    pick = np.sort(np.random.default_rng(5).choice(len(boxes), size=48, replace=False))
    ref = O.local_eigenvalues(prob, boxes[pick], 6)
    rel, null = O.eigenvalue_errors(lr["ev"][pick], ref)
    rel64, null64 = O.eigenvalue_errors(out["fp64"]["ev"][pick], ref)
    xr = out["fp64_ref"]["x"]
    err = np.linalg.norm(lr["x"] - xr) / np.linalg.norm(xr)
    err64 = np.linalg.norm(out["fp64"]["x"] - xr) / np.linalg.norm(xr)
    print(f"learned: eig rel {rel:.2e} null {null:.2e}, x err {err:.2e}; fp64: eig rel {rel64:.2e} "
          f"null {null64:.2e}, x err {err64:.2e}; fallbacks {lr['st']['fallbacks']}")
    assert rel64 <= 1e-6 and null64 <= 1e-9, (rel64, null64)
    assert rel <= 1e-6 and null <= 1e-9, (rel, null)
