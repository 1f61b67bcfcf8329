"""Golden fixtures of the oracle on the reference's own problems.

The reference ships no golden vectors and cannot be built here (PETSc, SLEPc
and MPI are absent), so these fixtures pin the NumPy oracle
(oracle/pmf_oracle.py) on the problems the reference's drivers run, with the
drivers' settings, the right-hand side normalised as they do (VecNormalize)
and rtol 1e-8:

  test_c_aniso8       src/test.c:7-55: constant k = (2, 1, 0.5), 8^3 unit cube,
                      the well source, -sd 2 -en_lv1 3 -en_lv2 2 (pure Neumann)
  expe_scal_cross16   src/Expe_scal.c:11-64: the cross field 10^cr with cr = 3,
                      16^3, the well source, -sd 2 -en_lv1 4 -en_lv2 4, and
                      p = 0 on x = 0 so that the iteration count is not
                      rounding-sensitive
  unit_cube_grf32     the 32^3 unit-cube GRF workload (sigma 2, correlation
                      0.1, seed 1, p = 0 on x = 1, f = 1), -sd 4 -en_lv1 4
                      -en_lv2 4 (4^3 subdomains of 8^3)

Each <name>.npz holds the options (JSON), the local eigenvalues eig1
(subdomains x en_lv1), the level-3 eigenvalues eig2 (ranks x en_lv2), the
level-3 matrix A3, one preconditioner application y_pc = B x_pc with x_pc
= pc_input(n) (standard normal, seed 11, not stored), the right-hand side b,
the PCG iteration count and solution x.

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pmf_oracle as O  # noqa: E402
from premixfem_b200 import fields  # noqa: E402


def _normalised(prob):
    return dict(prob, source=prob["source"] / np.linalg.norm(prob["source"]))


CASES = {
    "test_c_aniso8": (lambda: _normalised(fields.aniso_const(8, 8, 8)), dict(sd=2, en_lv1=3, en_lv2=2)),
    "expe_scal_cross16": (lambda: _normalised(dict(fields.cross(16, 3), dirichlet={"x-": 0.0})),
                          dict(sd=2, en_lv1=4, en_lv2=4)),
    "unit_cube_grf32": (lambda: fields.unit_cube_grf(32, seed=1), dict(sd=4, en_lv1=4, en_lv2=4)),
}


def pc_input(n):
    return np.random.default_rng(11).standard_normal(n)


def compute(name):
    make, opts = CASES[name]
    prob = make()
    r = O.solve(prob, O.Options(**opts))
    pc = r["pc"]
    return dict(options=json.dumps(opts), eig1=np.stack(pc.eigvals_lv1), eig2=np.stack(pc.eigvals_lv2), A3=pc.A3,
                y_pc=pc.apply(pc_input(r["op"].n)), b=r["b"], its=np.int64(r["its"]), x=r["x"])


def main():
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **compute(name))
        print("wrote", name)


if __name__ == "__main__":
    main()
