"""The CUDA path against the committed golden fixtures (tests/golden/).

The fixtures hold the oracle's results on the reference's own problems
(src/test.c, the cross field of src/Expe_scal.c) and on the 32^3 GRF
workload; this checks the library against them without running the oracle:
right-hand side 1e-13; local and level-3 eigenvalues 1e-6 relative with a
floor of 1e-9 x the largest of the subdomain (rank) for the zero modes; one
preconditioner application 1e-6 (problems with a Dirichlet face: without one,
the +NIL shift of the level-3 matrix amplifies the constant part of B x by
1e12, so B x itself is not comparable); PCG iterations +-1; the solution
within 1e-7 of the fixture's (two CG solutions at rtol 1e-8), modulo
constants for the pure-Neumann test.c problem.
"""
import importlib.util
import json
import os

import numpy as np
import pytest

from premixfem_b200.solver import DarcySolver, options_string

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "make_golden.py"))
G = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(G)


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def _eig_err(got, ref):
    scale = np.abs(ref).max(axis=1, keepdims=True)
    return float((np.abs(got - ref) / np.maximum(np.abs(ref), 1e-3 * scale)).max())


@pytest.mark.parametrize("name", sorted(G.CASES))
def test_library_matches_golden(native, name):
    ref = dict(np.load(os.path.join(HERE, name + ".npz")))
    make, opts = G.CASES[name]
    assert json.loads(str(ref["options"])) == opts
    prob = make()
    s = DarcySolver.from_problem(prob, options_string(opts))
    s.setup()
    b = s.rhs(prob["source"].ravel())
    assert _rel(b, ref["b"]) <= 1e-13
    ev1, _, _, status = s.eigen_lv1()
    assert (status != 1).all()
    assert _eig_err(ev1, ref["eig1"]) <= 1e-6
    ev3, _, _ = s.eigen_lv2()
    assert _eig_err(ev3, ref["eig2"]) <= 1e-6
    neumann = not prob["dirichlet"]
    if not neumann:
        y = s.pc_apply(G.pc_input(b.size))
        assert _rel(y, ref["y_pc"]) <= 1e-6
    x, its, _, reason = s.solve(b)
    s.close()
    assert reason == "converged"
    assert abs(its - int(ref["its"])) <= 1, (its, int(ref["its"]))
    xr = ref["x"]
    if neumann:
        x, xr = x - x.mean(), xr - xr.mean()
    assert _rel(x, xr) <= 1e-7
