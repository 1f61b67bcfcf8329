"""-ksp_constant_null_space on the GPU against the oracle.

With the option, PETSc's CG removes the operator's constant null space from
every preconditioned residual (KSP_PCApply -> MatNullSpaceRemove); the
right-hand side is not projected.  The case is the reference's own test.c
problem (src/test.c:7-38): constant k = (2, 1, 0.5), the well source, no
Dirichlet face, so A is singular.  Parity bars as for the other PCG tests:
iterations within +-1 of the oracle with the same option, the solution within
1e-8 relative of the zero-mean direct solve, compared modulo constants.
"""
import numpy as np
import pytest

from oracle import pmf_oracle as O
from premixfem_b200 import fields
from premixfem_b200.solver import DarcySolver, options_string

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_constant_null_space_matches_oracle(native, precision):
    prob = fields.aniso_const(8, 8, 8)
    d = {"sd": 2, "en_lv1": 4, "en_lv2": 4}
    ref = O.solve(prob, O.Options(**d, constant_null_space=True))
    assert ref["reason"] == "converged_rtol"
    s = DarcySolver.from_problem(prob, options_string(dict(d, pmf_precision=precision)) + " -ksp_constant_null_space")
    s.setup()
    b = s.rhs(prob["source"].ravel())
    x, its, rnorm, reason = s.solve(b)
    s.close()
    assert reason == "converged"
    assert abs(its - ref["its"]) <= 1, (its, ref["its"])
    assert rnorm <= 1e-8 * np.linalg.norm(b) * (1 + 1e-6)
    xd = O.direct_solve(ref["op"], ref["b"])
    xd = xd - xd.mean()
    err = np.linalg.norm((x - x.mean()) - xd) / np.linalg.norm(xd)
    assert err <= 1e-8, err


def test_constant_null_space_option_values(native):
    # PETSc boolean option: bare flag or a true/false word; anything else is an argument error
    from premixfem_b200._native import PmfError
    for opt in ("-ksp_constant_null_space", "-ksp_constant_null_space true", "-ksp_constant_null_space 0"):
        DarcySolver((1.0, 1.0, 1.0), (8, 8, 8), "-sd 2 " + opt).close()
    with pytest.raises(PmfError) as e:
        DarcySolver((1.0, 1.0, 1.0), (8, 8, 8), "-sd 2 -ksp_constant_null_space maybe")
    assert e.value.code == 62
