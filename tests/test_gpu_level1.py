"""The level-1 solve kernels with the subdomain-blocked IC(0) factor.

k_ic_apply_blk stages each subdomain's {tx, ty, tz, 1/D} block with one TMA
bulk copy and does the natural-order kernel k_ic_apply's arithmetic in the
same order; k_ic_apply_stg (-pmf_lv1_kernel staged) is the same solve with all
of a CTA's global loads (x, the iterate, the diagonal and the face halo)
issued in one unrolled pass before any is used.  The compiler contracts some
multiply-adds differently in the three, so a preconditioner application
agrees with the natural kernel's to 1e-12 in FP64 and 1e-5 in the mixed form,
the bars test_gpu_tune.py sets for the other launch-shape candidates.  Shapes:
16^3 subdomains of the fracture workload, ragged 16 x ny x nz subdomains with
Dirichlet faces on several sides, and several virtual ranks along x.  The PCG
solves agree to iterations +-1 and the solution to 1e-10 (FP64) / 1e-7
(mixed).  Device vectors at an odd 8-byte offset give the same result as
aligned ones, and a mesh a kernel cannot take is refused when it is forced.
"""
import numpy as np
import pytest

from premixfem_b200 import fields
from premixfem_b200._native import PmfError
from premixfem_b200.solver import DarcySolver, options_string

pytestmark = pytest.mark.gpu

CASES = {
    "fracture64_sd4": (lambda: fields.fracture256(64, seed=3), {"sd": 4, "en_lv1": 6, "en_lv2": 4}),
    "ragged_dirichlet": (lambda: fields.random_box((32, 40, 28), seed=3, sigma=2.0,
                                                   dirichlet={"y+": 0.0, "z-": 1.0}),
                         {"pmf_sd": (2, 3, 2), "en_lv1": 4, "en_lv2": 3}),
    "xranks": (lambda: fields.random_box((48, 32, 30), seed=4, sigma=1.5, dirichlet={"x+": 0.0}),
               {"pmf_sd": (1, 2, 2), "pmf_vranks": (3, 1, 1), "en_lv1": 4, "en_lv2": 2}),
}


def _solver(prob, d, kernel, precision):
    s = DarcySolver.from_problem(prob, options_string(dict(d, pmf_precision=precision, pmf_lv1_kernel=kernel)))
    s.setup()
    return s


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_blocked_level1_is_bit_identical(native, name, precision):
    mk, d = CASES[name]
    prob = mk()
    n = int(np.prod(prob["mesh"]))
    x = np.random.default_rng(9).standard_normal(n)
    out = {}
    for kernel in ("natural", "blocked", "staged"):
        s = _solver(prob, d, kernel, precision)
        y = s.pc_apply(x)
        b = s.rhs(prob["source"].ravel())
        xs, its, rnorm, reason = s.solve(b)
        s.close()
        assert reason == "converged"
        out[kernel] = (y, xs, its)
    tol_pc, tol_x = (1e-12, 1e-10) if precision == "fp64" else (1e-5, 1e-7)
    for kernel in ("blocked", "staged"):
        rel_pc = np.linalg.norm(out["natural"][0] - out[kernel][0]) / np.linalg.norm(out["natural"][0])
        assert rel_pc <= tol_pc, (kernel, rel_pc)
        assert abs(out["natural"][2] - out[kernel][2]) <= 1, kernel
        rel = np.linalg.norm(out["natural"][1] - out[kernel][1]) / np.linalg.norm(out["natural"][1])
        assert rel <= tol_x, (kernel, rel)


def test_blocked_level1_misaligned_device_vector(native):
    torch = pytest.importorskip("torch")
    mk, d = CASES["fracture64_sd4"]
    prob = mk()
    n = int(np.prod(prob["mesh"]))
    x = np.random.default_rng(2).standard_normal(n)
    s = _solver(prob, d, "blocked", "mixed")
    ref = s.pc_apply(x)
    buf = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(x).cuda()
    xo = buf[1:]  # 8 bytes past a 16-byte boundary
    yo = torch.empty(n + 1, dtype=torch.float64, device="cuda")[1:]
    s.pc_apply(xo, yo)
    s.close()
    assert np.array_equal(yo.cpu().numpy(), ref)


def test_blocked_level1_refused_where_it_does_not_fit(native):
    prob = fields.unit_cube_grf(16, seed=1)  # 8^3 subdomains
    s = DarcySolver.from_problem(prob, "-sd 2 -pmf_lv1_kernel blocked")
    with pytest.raises(PmfError) as e:
        s.setup()
    assert e.value.code == 56
    s.close()


def test_staged_level1_refused_where_it_does_not_fit(native):
    # 16 x 8 x 32 subdomains: the blocked kernel takes them (256 x-lines), the
    # staged one does not (nz > 16)
    prob = fields.random_box((32, 16, 64), seed=5, sigma=1.0, dirichlet={"x-": 1.0})
    s = DarcySolver.from_problem(prob, "-sd 2 -pmf_lv1_kernel blocked")
    s.setup()
    s.close()
    s = DarcySolver.from_problem(prob, "-sd 2 -pmf_lv1_kernel staged")
    with pytest.raises(PmfError) as e:
        s.setup()
    assert e.value.code == 56
    s.close()
