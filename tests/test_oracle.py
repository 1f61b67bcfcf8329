"""Known-answer pins of the CPU oracle (no GPU).

The reference ships no golden vectors and cannot be built here, so the oracle
is pinned to closed-form mathematics instead (parity with the reference
itself stays unpinned):
  * constant-coefficient 7-point operators have Kronecker-sum spectra;
  * the MEAN mass matrix of a constant field is a multiple of the identity,
    so the local GHEP spectrum is the Neumann Laplacian's;
  * IC(0) of the 7-point pattern equals the textbook pattern-restricted IC(0)
    and is exact on a 1-D chain;
  * PCG reaches the direct solution; the V-cycle is symmetric positive definite.
"""
import numpy as np
import pytest
import scipy.linalg as sla

from oracle import pmf_oracle as O
from premixfem_b200 import fields


def lap1d_neumann_eigs(n):
    return 2.0 - 2.0 * np.cos(np.pi * np.arange(n) / n)


def test_split_matches_reference_rule():
    # src/PreMixFEM_3D.c:62-71: first n % sd parts get one more cell
    assert O.split(10, 3) == ([0, 4, 7], [4, 3, 3])
    assert O.split(16, 4) == ([0, 4, 8, 12], [4, 4, 4, 4])
    assert O.split(7, 7) == (list(range(7)), [1] * 7)
    s, l = O.split(257, 16)
    assert sum(l) == 257 and l[0] == 17 and l[1] == 16


def test_options_reset_sd_one_to_two():
    assert O.Options(sd=1).normalized().sd == (2, 2, 2)  # :1718-1721
    assert O.Options(si_lv1=0).normalized().si_lv1 == 1


def test_operator_constant_kappa_spectrum():
    M, N, P = 4, 3, 5
    prob = fields.aniso_const(M, N, P)
    op = O.Operator(prob)
    kx, ky, kz = 2.0, 1.0, 0.5
    Hx, Hy, Hz = 1.0 / M, 1.0 / N, 1.0 / P
    tx = (Hy * Hz) ** 2 / (Hx * Hy * Hz) * kx
    ty = (Hz * Hx) ** 2 / (Hx * Hy * Hz) * ky
    tz = (Hx * Hy) ** 2 / (Hx * Hy * Hz) * kz
    ex = (tz * lap1d_neumann_eigs(P)[:, None, None] + ty * lap1d_neumann_eigs(N)[None, :, None]
          + tx * lap1d_neumann_eigs(M)[None, None, :]).ravel()
    ev = np.linalg.eigvalsh(op.A.toarray())
    np.testing.assert_allclose(np.sort(ev), np.sort(ex), rtol=1e-12, atol=1e-12 * ex.max())


def test_operator_harmonic_mean_and_symmetry():
    prob = fields.random_box((5, 4, 3), seed=3, sigma=2.0)
    op = O.Operator(prob)
    A = op.A.toarray()
    np.testing.assert_allclose(A, A.T, rtol=0, atol=0)
    kx = prob["kappa"][0]
    H = op.H
    c = (H[1] * H[2]) ** 2 / (H[0] * H[1] * H[2])
    # face between (0,0,0) and (1,0,0)
    t = c * 2.0 / (1.0 / kx[0, 0, 0] + 1.0 / kx[0, 0, 1])
    assert A[0, 1] == -t
    # rows sum to the Dirichlet term only (x- face is Dirichlet here)
    rs = A.sum(axis=1).reshape(op.mesh[2], op.mesh[1], op.mesh[0])
    np.testing.assert_allclose(rs, op.db, rtol=1e-12, atol=1e-12 * np.abs(A).max())


def test_ic0_recurrence_equals_textbook_ic0():
    prob = fields.random_box((4, 3, 3), seed=5, sigma=1.5)
    op = O.Operator(prob)
    A = op.principal((0, 4, 0, 3, 0, 3)).toarray()
    L = O.ic0_general(A)
    D = O.ic0_pivots(A)
    np.testing.assert_allclose(np.diag(L) ** 2, D, rtol=1e-13)
    Lo = np.tril(A, -1)
    F = (np.diag(D) + Lo) @ np.diag(1.0 / D) @ (np.diag(D) + Lo.T)
    np.testing.assert_allclose(F, L @ L.T, rtol=1e-12, atol=1e-12 * np.abs(A).max())


def test_ic0_exact_on_chain():
    prob = fields.random_box((9, 1, 1), seed=2)
    op = O.Operator(prob)
    A = op.A
    sol = O.IC0Solver(A)
    b = np.random.default_rng(0).standard_normal(9)
    np.testing.assert_allclose(A @ sol.solve(b), b, rtol=1e-12, atol=1e-12)


def test_local_ghep_mean_constant_field_is_laplacian():
    M = N = P = 8
    prob = fields.aniso_const(M, N, P)
    op = O.Operator(prob)
    box = (0, 4, 4, 4, 0, 4)
    An = op.neumann(box).toarray()
    Md = op.mass_diag(box, O.EIG_OP_MEAN)
    np.testing.assert_allclose(Md, 3.5)
    w = sla.eigh(An, np.diag(Md), eigvals_only=True)
    Hx, Hy, Hz = 1.0 / M, 1.0 / N, 1.0 / P
    meas = Hx * Hy * Hz
    tx = (Hy * Hz) ** 2 / meas * 2.0
    ty = (Hz * Hx) ** 2 / meas * 1.0
    tz = (Hx * Hy) ** 2 / meas * 0.5
    e = lap1d_neumann_eigs(4)
    ex = (tz * e[:, None, None] + ty * e[None, :, None] + tx * e[None, None, :]).ravel() / 3.5
    np.testing.assert_allclose(np.sort(w), np.sort(ex), rtol=1e-10, atol=1e-10 * ex.max())


def test_mod_mass_quirk():
    # constant kappa, interior subdomain: x-row cells get the right face twice
    # except the last one; the first also gets its left face (:258-274).
    M = N = P = 8
    k = np.ones((P, N, M))
    prob = {"mesh": (M, N, P), "dom": (1.0, 1.0, 1.0), "kappa": (k, k, k), "source": np.zeros((P, N, M)),
            "dirichlet": {}}
    op = O.Operator(prob)
    box = (2, 4, 2, 4, 2, 4)
    Md = op.mass_diag(box, O.EIG_OP_MOD).reshape(4, 4, 4)
    h2 = (1.0 / 8) ** 2
    unit = 2.0 / h2 * (1.0 / 8) ** 3  # 2*avg/H^2 * |K|
    # y and z contribute 2 faces each; x: first cell 3, middle 2, last 1
    np.testing.assert_allclose(Md[1, 1, :], unit * np.array([4 + 3, 4 + 2, 4 + 2, 4 + 1]))


def test_pcg_matches_direct_and_counts_iterations():
    prob = fields.unit_cube_grf(16, seed=1)
    res = O.solve(prob, O.Options(sd=2, en_lv1=4, en_lv2=4))
    op = res["op"]
    xd = O.direct_solve(op, res["b"])
    assert res["reason"] == "converged_rtol"
    assert 5 <= res["its"] <= 60
    assert np.linalg.norm(res["x"] - xd) / np.linalg.norm(xd) < 1e-7
    assert res["hist"][-1] <= 1e-8 * res["hist"][0]


def test_vcycle_is_spd():
    prob = fields.unit_cube_grf(8, seed=2)
    op = O.Operator(prob)
    pc = O.Preconditioner(op, O.Options(sd=2, en_lv1=3, en_lv2=2))
    rng = np.random.default_rng(1)
    x, y = rng.standard_normal(op.n), rng.standard_normal(op.n)
    a, b = y @ pc.apply(x), x @ pc.apply(y)
    assert abs(a - b) <= 1e-10 * max(abs(a), abs(b))
    assert x @ pc.apply(x) > 0


@pytest.mark.parametrize("w_cycle", [False, True])
def test_vranks_reproduce_multi_rank_structure(w_cycle):
    prob = fields.unit_cube_grf(16, seed=1)
    res = O.solve(prob, O.Options(sd=2, vranks=(2, 1, 2), en_lv1=4, en_lv2=3, use_W_cycle=w_cycle))
    pc = res["pc"]
    assert len(pc.lay.ranks) == 4 and len(pc.lay.subs) == 32
    assert pc.A3.shape == (12, 12)
    assert res["reason"] == "converged_rtol"


def test_constant_null_space_steadies_pure_neumann_cg():
    # Pure Neumann, default +NIL shift of the level-3 matrix: the constant mode
    # of z is amplified by 1/NIL, so the plain iteration count at 1e-10 moves
    # with 1e-15 perturbations of the source.  Removing the constant from z
    # (-ksp_constant_null_space) makes it deterministic, and every run reaches
    # the zero-mean direct solution.
    opts = dict(sd=2, vranks=(1, 2, 2), en_lv1=4, en_lv2=4, rtol=1e-10, constant_null_space=True)
    rng = np.random.default_rng(0)
    its = set()
    for t in range(4):
        prob = fields.cross(16, 3)
        src = prob["source"] * (1 + (1e-15 * rng.standard_normal(prob["source"].shape) if t else 0.0))
        prob["source"] = src / np.linalg.norm(src)
        r = O.solve(prob, O.Options(**opts))
        assert r["reason"] == "converged_rtol"
        its.add(r["its"])
        xd = O.direct_solve(r["op"], r["b"])
        xd -= xd.mean()
        assert np.linalg.norm(r["x"] - r["x"].mean() - xd) <= 1e-9 * np.linalg.norm(xd)
    assert len(its) == 1, its


@pytest.mark.parametrize("contrast,mesh,sd,its", [(1e6, (20, 30, 10), (2, 3, 2), 76), (1e4, (20, 20, 10), (2, 2, 2), 43)])
def test_fp32_stored_basis_keeps_the_channel_iterations(contrast, mesh, sd, its):
    # The mixed form stores the local eigenvectors in FP32.  On the layered
    # channel fields, exact eigenvectors rounded to FP32 give the iteration
    # count of the FP64 ones: the storage is not what limits the mixed form there.
    M, N, P = mesh
    prob = fields.layered(seed=2, M=M, N=N, P=P, smooth_layers=4, contrast=contrast)
    opts = dict(sd=sd, en_lv1=4, en_lv2=4, constant_null_space=True)
    r64 = O.solve(prob, O.Options(**opts))
    r32 = O.solve(prob, O.Options(**opts, phi_fp32=True))
    assert r64["reason"] == r32["reason"] == "converged_rtol"
    assert r64["its"] == its and abs(r32["its"] - r64["its"]) <= 1


def test_channel_subdomains_hold_near_zero_clusters():
    # The mechanism behind the channel-field stalls of a loose eigen stopping
    # test: every separate channel piece in a subdomain gives a near-zero local
    # mode, so many subdomains hold clusters of eigenvalues far below lscale
    # (max diag(A_N) / M), and the en_lv1 cut falls inside some of them.
    prob = fields.layered(seed=2, M=30, N=20, P=15, smooth_layers=6)
    o = O.Options(sd=(3, 2, 3), en_lv1=8, en_lv2=4)
    op = O.Operator(prob)
    pc = O.Preconditioner(op, o)
    ev = np.stack(pc.eigvals_lv1)
    lscale = np.array([(np.diag(op.neumann(s).toarray()) / op.mass_diag(s, o.eg_op)).max() for s in pc.lay.subs])
    near_zero = (ev / lscale[:, None] < 1e-4).sum(axis=1)
    assert (near_zero >= 2).sum() >= 5
    assert near_zero.max() > 4  # a cluster straddling en_lv1 = 4
