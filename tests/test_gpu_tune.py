"""The launch-shape tuner: every candidate it may pick computes the same thing.

The tuner chooses by speed alone, so each candidate launch shape is checked
here by forcing it (PMF_TUNE_FORCE=c): the network forward pass of each row
tile, and of the tcgen05 convolution (candidate 4, the 3x3x3 layers on 16^3
patches; the other layers clamp to their last tile), against the CPU oracle
(2e-2, the forward-pass tolerance of test_gpu_net.py), and the preconditioner application with each thread count
of the level-1 solve and the level-2 restriction / prolongation against the
built-in shape (1e-12 in FP64, 1e-5 in mixed precision: only the order of the
block reductions changes).  The report of a tuned set-up lists its choices.
"""
import ctypes as C
import json

import numpy as np
import pytest

from oracle import net_oracle as NO
from premixfem_b200 import _native, fields, learned
from premixfem_b200.solver import DarcySolver, options_string

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


@pytest.mark.parametrize("cand", [0, 1, 2, 3, 4])
def test_net_forward_every_tile(native, monkeypatch, cand):
    torch = pytest.importorskip("torch")
    monkeypatch.setenv("PMF_TUNE_FORCE", str(cand))
    net = learned.Net(seed=7)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2, 16, 16, 16, 16)).astype(np.float32)
    x[..., 5:] = 0.0
    xt = torch.from_numpy(x).to(torch.bfloat16).cuda()
    xb = xt.float().cpu().numpy().astype(np.float64)
    W, b = [], []
    for l in range(9):
        w_, b_ = net.weights(l)
        W.append(w_.astype(np.float64))
        b.append(b_.astype(np.float64))
    y = torch.empty((2, 4096, 16), dtype=torch.float32, device="cuda")
    net.forward(xt, y)
    torch.cuda.synchronize()
    ref = NO.forward(xb, W, b, bf16=True)[-1].reshape(2, 4096, 16)
    assert _rel(y.cpu().numpy(), ref) < 2e-2


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pc_apply_every_thread_shape(native, monkeypatch, precision):
    prob = fields.fracture256(64, seed=3)
    opts = options_string({"sd": 4, "en_lv1": 6, "en_lv2": 4, "pmf_precision": precision})
    x = np.random.default_rng(5).standard_normal(64 ** 3)
    out = []
    # level 1 with an iterate: the natural kernel at 256 / 384 / 512 / 768 / 1024
    # threads, the blocked kernel at 512 / 256 and the staged one; the first
    # visit: natural, blocked 512 / 256, staged (cand 4 and up clamp to it);
    # the restriction / prolongation's three shapes (others clamped)
    for cand in range(8):
        monkeypatch.setenv("PMF_TUNE_FORCE", str(cand))
        s = DarcySolver.from_problem(prob, opts)
        s.setup()
        out.append(s.pc_apply(x))
        s.close()
    tol = 1e-12 if precision == "fp64" else 1e-5
    for cand in range(1, 8):
        assert _rel(out[cand], out[0]) <= tol, (cand, _rel(out[cand], out[0]))


def test_report_lists_the_tuned_shapes(native, monkeypatch):
    monkeypatch.delenv("PMF_TUNE_FORCE", raising=False)
    lib = _native.load()
    prob = fields.unit_cube_grf(32, seed=2)
    s = DarcySolver.from_problem(prob, "-sd 4 -pmf_autotune 1")
    s.setup()
    s.close()
    n = lib.pmf_tune_report(None, 0)
    buf = C.create_string_buffer(n + 1)
    assert lib.pmf_tune_report(buf, n + 1) == n
    table = json.loads(buf.value.decode())
    # 32^3 with -sd 4: 64 subdomains of 8^3 cells (64 x-lines each), 4 eigenvectors
    shapes = ("ic_apply|f64|n64|c512|l64|", "resid_restrict|f64|n64|c512|k4|", "prolong|f64|n64|c512|k4|")
    keys = [k for k in table if k.startswith(shapes)]
    assert len(keys) == 3, list(table)
    for k in keys:
        e = table[k]
        assert 0 <= e["choice"] < len(e["us"])
        assert e["us"][e["choice"]] == min(t for t in e["us"] if t >= 0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_eigensolver_every_online_shape(native, monkeypatch, precision):
    """The lock-step eigensolver's online candidates (preconditioner column batch
    3 / 8 / 1, update tiles <6,1> / <8,2>, each with one or two groups of cells
    loading ahead, and the CUDA-core update) give the same local eigenvalues
    (1e-6 relative) and the same PCG iteration count (+-1)."""
    prob = fields.fracture256(64, seed=3)
    opts = options_string({"sd": 4, "en_lv1": 6, "en_lv2": 4, "pmf_precision": precision})
    res = []
    for cand in (0, 1, 2, 3, 4):
        monkeypatch.setenv("PMF_TUNE_FORCE", str(cand))
        s = DarcySolver.from_problem(prob, opts)
        s.setup()
        ev = s.eigen_lv1()[0].copy()
        b = s.rhs(prob["source"].ravel())
        _, its, _, reason = s.solve(b)
        assert reason == "converged"
        res.append((ev, its))
        s.close()
    for cand in (1, 2, 3, 4):
        ev0, ev = res[0][0], res[cand][0]
        rel = np.abs(ev - ev0) / np.maximum(np.abs(ev0), 1e-9 * np.abs(ev0).max())
        assert rel.max() <= 1e-6, (cand, rel.max())
        assert abs(res[cand][1] - res[0][1]) <= 1, (cand, res[cand][1], res[0][1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_every_pcg_kernel(native, monkeypatch, precision):
    """The three candidates of the CG step's fused p-update + operator kernel
    (one cell per thread, the 2.5-D march, the grid-stride kernel; forced
    together with the other shapes' candidates 0 / 1 / 2) converge in the same
    number of iterations (+-1) to the same solution (1e-7 relative: only the
    order of the dot-product partial sums differs)."""
    prob = fields.fracture256(64, seed=3)
    opts = options_string({"sd": 4, "en_lv1": 6, "en_lv2": 4, "pmf_precision": precision})
    res = []
    for cand in (0, 1, 2):
        monkeypatch.setenv("PMF_TUNE_FORCE", str(cand))
        s = DarcySolver.from_problem(prob, opts)
        s.setup()
        b = s.rhs(prob["source"].ravel())
        x, its, _, reason = s.solve(b)
        assert reason == "converged"
        res.append((x.copy(), its))
        s.close()
    for cand in (1, 2):
        assert abs(res[cand][1] - res[0][1]) <= 1, (cand, res[0][1], res[cand][1])
        assert _rel(res[cand][0], res[0][0]) <= 1e-7, (cand, _rel(res[cand][0], res[0][0]))
