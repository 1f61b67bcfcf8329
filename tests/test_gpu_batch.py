"""A batch of independent problems set up and solved together on the GPU.

The batching workload's distribution (per-axis sizes drawn from a range,
exp-GRF fields with their own sigma and correlation, p = 0 on x = 1, ragged
8^3 tiles, k = 4, four right-hand sides: the unit source and three N(0,1)
fields) at reduced sizes, against the oracle run problem by problem with the
same partition (one rank per problem, as one reference run per problem):
local eigenvalues of every subdomain (FP64), and for every problem and
right-hand side the PCG iteration count (+-1) and the solution (1e-8 relative
of the oracle's).
"""
import numpy as np
import pytest

from oracle import pmf_oracle as O
from premixfem_b200 import fields
from premixfem_b200.solver import BatchSolver, options_string

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_ref():
    batch = fields.grf_batch(count=4, seed=3, lo=10, hi=26)
    refs = []
    for prob, sources in batch:
        sd = fields.tiles(prob["mesh"])
        op = O.Operator(prob)
        pc = O.Preconditioner(op, O.Options(sd=sd, en_lv1=4, en_lv2=4))
        sols = []
        for src in sources:
            b = O.Operator(dict(prob, source=src)).rhs()
            x, its, _, reason = O.pcg(op.A, b, pc.apply)
            assert reason == "converged_rtol"
            sols.append((x, its))
        refs.append((sd, pc, sols))
    return batch, refs


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_oracle_per_problem(native, batch_ref, precision):
    batch, refs = batch_ref
    problems = [p for p, _ in batch]
    s = BatchSolver(problems, [r[0] for r in refs], options_string({"en_lv1": 4, "en_lv2": 4,
                                                                    "pmf_precision": precision}))
    s.set_kappa_problems(problems)
    s.setup()
    if precision == "fp64":
        ev, ks, iters, status = s.eigen_lv1()
        ref_ev = np.concatenate([np.stack(r[1].eigvals_lv1) for r in refs])
        scale = np.abs(ref_ev).max(axis=1, keepdims=True)
        err = np.abs(ev - ref_ev) / np.maximum(np.abs(ref_ev), 1e-3 * scale)
        assert err.max() <= 1e-6, err.max()
    for j in range(4):
        b = s.rhs(s.pack([srcs[j] for _, srcs in batch]))
        x, its, rnorm, reasons = s.solve(b)
        xs = s.unpack(x)
        for q, (prob, _) in enumerate(batch):
            x_ref, its_ref = refs[q][2][j]
            assert reasons[q] == "converged", (q, j, reasons[q])
            assert abs(int(its[q]) - its_ref) <= 1, (q, j, int(its[q]), its_ref)
            rel = np.linalg.norm(xs[q] - x_ref) / np.linalg.norm(x_ref)
            assert rel <= 1e-8, (q, j, rel)
    s.close()


def test_batch_rejects_single_problem_calls(native):
    """The single-problem CG and Dirichlet calls refuse a batch (73)."""
    from premixfem_b200._native import PmfError
    from premixfem_b200.solver import DarcySolver
    batch = fields.grf_batch(count=2, seed=5, lo=10, hi=12)
    problems = [p for p, _ in batch]
    s = BatchSolver(problems, [fields.tiles(p["mesh"]) for p in problems], "-en_lv1 3")
    s.set_kappa_problems(problems)
    s.setup()
    b = s.rhs(s.pack([srcs[0] for _, srcs in batch]))
    with pytest.raises(PmfError) as e:
        DarcySolver.solve(s, b)
    assert e.value.code == 73
    with pytest.raises(PmfError) as e:
        DarcySolver.set_dirichlet(s, "x-", 1.0)
    assert e.value.code == 73
    s.close()
