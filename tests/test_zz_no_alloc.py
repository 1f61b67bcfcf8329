"""pmf_residual_noalloc against the existing pmf_apply_A entry point.

Collected last on purpose (file name), so it runs both after the other GPU
tests and, when selected alone, in a fresh process.  Two calls in a row check
that the static scratch is left ready (ticket back at zero) by each call.
Tolerances: r within 1e-14 relative L2 of b - A x formed from pmf_apply_A
(the same stencil arithmetic; only the subtraction order may differ), and
||r|| within 1e-12 relative of the norm of that vector.
"""
import ctypes as C

import numpy as np
import pytest

from premixfem_b200 import _native, fields
from premixfem_b200.solver import DarcySolver

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_residual_noalloc_matches_apply_A_twice(native):
    torch = pytest.importorskip("torch")
    prob = fields.random_box((37, 29, 23), seed=11, sigma=2.0, dirichlet={"x-": 1.0})
    s = DarcySolver.from_problem(prob, "-sd 2")
    s.setup()
    n = 37 * 29 * 23
    rng = np.random.default_rng(4)
    stream = torch.cuda.current_stream()
    for call in range(2):
        b = rng.standard_normal(n)
        x = rng.standard_normal(n)
        ref_r = b - s.apply_A(x)
        bd = torch.from_numpy(b).cuda()
        xd = torch.from_numpy(x).cuda()
        rd = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        nd = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = native.pmf_residual_noalloc(s.h, _ptr(bd), _ptr(xd), _ptr(rd), _ptr(nd),
                                         C.c_void_p(stream.cuda_stream))
        assert rc == 0, native.pmf_last_error()
        torch.cuda.synchronize()
        r = rd.cpu().numpy()
        rn = float(nd.cpu().numpy()[0])
        assert np.linalg.norm(r - ref_r) <= 1e-14 * np.linalg.norm(ref_r), f"call {call}"
        assert abs(rn - np.linalg.norm(ref_r)) <= 1e-12 * np.linalg.norm(ref_r), f"call {call}"
    s.close()


def test_residual_noalloc_rejects_meshes_beyond_limit(native):
    # The size check comes before any device work; creating the handle
    # allocates no mesh-sized device memory.
    s = DarcySolver((1.0, 1.0, 1.0), (512, 256, 257), "-sd 2")
    null = C.c_void_p(0)
    rc = native.pmf_residual_noalloc(s.h, null, null, null, null, null)
    assert rc == 62
    assert b"PMF_NOALLOC_MAX_CELLS" in native.pmf_last_error()
    s.close()
