"""CPU checks of the network oracle (no GPU): its gradients against finite
differences on a small network of the same layer kinds, the subspace loss
gradient, and the bfloat16 rounding."""
import numpy as np

from oracle import net_oracle as NO

TINY = [
    (NO.CONV3, 2, 4, 4, 4, 1, -1, 0, 1),
    (NO.DOWN2, 4, 6, 4, 2, 1, -1, 1, 2),
    (NO.CONV3, 6, 6, 2, 2, 1, -1, 2, 3),
    (NO.UP2, 6, 4, 2, 4, 1, 1, 3, 4),
    (NO.CONV1, 4, 3, 4, 4, 0, -1, 4, 5),
]


def _tiny_params(rng):
    W = [rng.standard_normal((NO.taps(l[0]), l[1], l[2])) * 0.5 for l in TINY]
    b = [rng.standard_normal(l[2]) * 0.1 for l in TINY]
    return W, b


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    W, b = _tiny_params(rng)
    x = rng.standard_normal((2, 4, 4, 4, 2))
    R = rng.standard_normal((2, 4, 4, 4, 3))

    def f(W_):
        return float(np.sum(NO.forward(x, W_, b, TINY)[-1] * R))

    acts = NO.forward(x, W, b, TINY)
    dW, db = NO.backward(acts, W, R, TINY)
    h = 1e-6
    for li in range(len(TINY)):
        for _ in range(4):
            idx = tuple(rng.integers(0, s) for s in W[li].shape)
            Wp = [w.copy() for w in W]
            Wm = [w.copy() for w in W]
            Wp[li][idx] += h
            Wm[li][idx] -= h
            fd = (f(Wp) - f(Wm)) / (2 * h)
            assert abs(fd - dW[li][idx]) <= 1e-5 * max(1.0, abs(fd)), (li, idx, fd, dW[li][idx])
    # bias of the first layer
    bp = [v.copy() for v in b]
    bm = [v.copy() for v in b]
    bp[0][1] += h
    bm[0][1] -= h
    fd = (np.sum(NO.forward(x, W, bp, TINY)[-1] * R) - np.sum(NO.forward(x, W, bm, TINY)[-1] * R)) / (2 * h)
    assert abs(fd - db[0][1]) <= 1e-5 * max(1.0, abs(fd))


def test_subspace_loss_gradient_and_invariance():
    rng = np.random.default_rng(1)
    B, n, k = 2, 64, 3
    y = rng.standard_normal((B, n, 4))
    V = rng.standard_normal((B, n, k))
    M = rng.uniform(0.5, 2.0, (B, n))
    loss, dy = NO.subspace_loss(y, V, M, k)
    h = 1e-6
    for _ in range(6):
        b_, v_, c_ = rng.integers(0, B), rng.integers(0, n), rng.integers(0, k)
        yp, ym = y.copy(), y.copy()
        yp[b_, v_, c_] += h
        ym[b_, v_, c_] -= h
        fd = (NO.subspace_loss(yp, V, M, k)[0].mean() - NO.subspace_loss(ym, V, M, k)[0].mean()) / (2 * h)
        assert abs(fd - dy[b_, v_, c_]) <= 1e-4 * max(1e-3, abs(fd))
    # only the span of the k predicted vectors matters
    Q = rng.standard_normal((k, k))
    y2 = y.copy()
    y2[:, :, :k] = y[:, :, :k] @ Q
    assert np.allclose(NO.subspace_loss(y2, V, M, k)[0], loss, rtol=1e-6)
    # a perfect prediction has zero loss
    yv = np.zeros_like(y)
    yv[:, :, :k] = V @ Q
    assert NO.subspace_loss(yv, V, M, k)[0].max() < 1e-8 * loss.mean()  # only the 1e-6 ridge remains


def test_bf16_rounding():
    vals = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 1e-3, 65504.0])
    r = NO.bf16_round(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0  # halfway between 1 and 1+2^-7: ties to even
    assert r[2] == 1.0078125
    assert abs(r[3] - (-3.140625)) < 1e-12
    assert abs(r[4] - 1e-3) / 1e-3 < 4e-3
    assert NO.bf16_round(r).tolist() == r.tolist()


def test_library_table_matches_oracle_table():
    """The layer table compiled into the library equals the oracle's (no GPU needed)."""
    from premixfem_b200 import learned
    got = learned.Net.layers()
    for (typ, cin, cout, si, so, taps), ref in zip(got, NO.LAYERS):
        assert (typ, cin, cout, si, so) == ref[:5]
        assert taps == NO.taps(typ)
