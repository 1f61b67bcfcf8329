"""CPU oracle of the learned-initialisation network and its subspace loss.

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the library.  The
network has no counterpart in the reference (the reference starts SLEPc from
its default vectors); this restates, in float64 NumPy, exactly what
premixfem_b200/csrc/k_net.cu computes, so the GPU forward pass, the GPU
gradients and the loss can be checked.  Layout: activations [B][z][y][x][c],
weights W[tap][cin][cout], tap = (dz+1)*9 + (dy+1)*3 + (dx+1) for 3x3x3
convolutions and dz*4 + dy*2 + dx for the 2x2x2 down/up layers.

`bf16=True` rounds every stored activation and the weights to bfloat16
(round to nearest even), as the GPU stores them, so that the comparison only
sees accumulation-order differences.
"""
from __future__ import annotations

import numpy as np

CONV3, DOWN2, UP2, CONV1 = 0, 1, 2, 3

# (type, cin, cout, s_in, s_out, relu, skip_act, in_act, out_act): the library's table
LAYERS = [
    (CONV3, 16, 32, 16, 16, 1, -1, 0, 1),
    (DOWN2, 32, 64, 16, 8, 1, -1, 1, 2),
    (CONV3, 64, 64, 8, 8, 1, -1, 2, 3),
    (DOWN2, 64, 96, 8, 4, 1, -1, 3, 4),
    (CONV3, 96, 96, 4, 4, 1, -1, 4, 5),
    (UP2, 96, 64, 4, 8, 1, 3, 5, 6),
    (UP2, 64, 32, 8, 16, 1, 1, 6, 7),
    (CONV3, 32, 32, 16, 16, 1, -1, 7, 8),
    (CONV1, 32, 16, 16, 16, 0, -1, 8, 9),
]


def taps(t):
    return 27 if t == CONV3 else (1 if t == CONV1 else 8)


def bf16_round(a):
    """Round float64/float32 values to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _shift3(x, dz, dy, dx):
    """x[b, z+dz, y+dy, x+dx] with zero outside (same spatial size)."""
    B, S = x.shape[0], x.shape[1]
    out = np.zeros_like(x)
    zs, ys, xs = slice(max(0, -dz), S - max(0, dz)), slice(max(0, -dy), S - max(0, dy)), slice(max(0, -dx), S - max(0, dx))
    zi, yi, xi = slice(max(0, dz), S + min(0, dz)), slice(max(0, dy), S + min(0, dy)), slice(max(0, dx), S + min(0, dx))
    out[:, zs, ys, xs] = x[:, zi, yi, xi]
    return out


def _offsets(t):
    return t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1  # dz, dy, dx


def layer_forward(typ, x, W, b):
    """Pre-activation output of one layer (float64)."""
    B, S = x.shape[0], x.shape[1]
    if typ == CONV3:
        out = np.zeros((B, S, S, S, W.shape[2]))
        for t in range(27):
            dz, dy, dx = _offsets(t)
            out += _shift3(x, dz, dy, dx) @ W[t]
    elif typ == DOWN2:
        so = S // 2
        out = np.zeros((B, so, so, so, W.shape[2]))
        for t in range(8):
            dz, dy, dx = t >> 2, (t >> 1) & 1, t & 1
            out += x[:, dz::2, dy::2, dx::2] @ W[t]
    elif typ == UP2:
        so = 2 * S
        out = np.zeros((B, so, so, so, W.shape[2]))
        for t in range(8):
            dz, dy, dx = t >> 2, (t >> 1) & 1, t & 1
            out[:, dz::2, dy::2, dx::2] = x @ W[t]
    else:
        out = x @ W[0]
    return out + b


def layer_backward(typ, x, W, dz_):
    """(dW, db, dx) of one layer given the pre-activation output gradient."""
    B, S = x.shape[0], x.shape[1]
    cin, cout = W.shape[1], W.shape[2]
    dW = np.zeros_like(W)
    dx = np.zeros_like(x)
    db = dz_.reshape(-1, cout).sum(0)
    if typ == CONV3:
        for t in range(27):
            oz, oy, ox = _offsets(t)
            xs = _shift3(x, oz, oy, ox)
            dW[t] = xs.reshape(-1, cin).T @ dz_.reshape(-1, cout)
            dx += _shift3(dz_ @ W[t].T, -oz, -oy, -ox)
    elif typ == DOWN2:
        for t in range(8):
            oz, oy, ox = t >> 2, (t >> 1) & 1, t & 1
            dW[t] = x[:, oz::2, oy::2, ox::2].reshape(-1, cin).T @ dz_.reshape(-1, cout)
            dx[:, oz::2, oy::2, ox::2] = dz_ @ W[t].T
    elif typ == UP2:
        for t in range(8):
            oz, oy, ox = t >> 2, (t >> 1) & 1, t & 1
            g = dz_[:, oz::2, oy::2, ox::2]
            dW[t] = x.reshape(-1, cin).T @ g.reshape(-1, cout)
            dx += g @ W[t].T
    else:
        dW[0] = x.reshape(-1, cin).T @ dz_.reshape(-1, cout)
        dx = dz_ @ W[0].T
    return dW, db, dx


def forward(x, weights, biases, layers=LAYERS, bf16=False):
    """All activations (list indexed like the library's act buffers); acts[-1] is the FP32-kind output."""
    rnd = bf16_round if bf16 else (lambda a: a)
    acts = [rnd(x)]
    acts += [None] * len(layers)
    for li, (typ, cin, cout, si, so, relu, skip, ia, oa) in enumerate(layers):
        W = rnd(weights[li])
        z = layer_forward(typ, acts[ia], W, biases[li])
        if skip >= 0:
            z = z + acts[skip]
        if relu:
            z = np.maximum(z, 0.0)
        acts[oa] = z if li == len(layers) - 1 else rnd(z)
    return acts


def backward(acts, weights, dy, layers=LAYERS, bf16=False):
    """Gradients (dW list, db list) for dL/dy given the activations of forward()."""
    rnd = bf16_round if bf16 else (lambda a: a)
    L = len(layers)
    dpre = [None] * L
    dW = [None] * L
    db = [None] * L
    dpre[L - 1] = dy
    for li in range(L - 1, -1, -1):
        typ, cin, cout, si, so, relu, skip, ia, oa = layers[li]
        gw, gb, gx = layer_backward(typ, acts[ia], rnd(weights[li]), dpre[li])
        dW[li], db[li] = gw, gb
        if li == 0:
            break
        for lj, lay in enumerate(layers):
            if lay[6] == ia:
                gx = gx + dpre[lj]
        gx = gx * (acts[ia] > 0)
        # the previous layer in the chain produces act ia
        prev = [lj for lj, lay in enumerate(layers) if lay[8] == ia][0]
        dpre[prev] = gx
    return dW, db


def subspace_loss(y, V, M, k):
    """Per-sample loss ||V - Y C||_M^2 / k with C = (Y^T M Y + eps I)^-1 Y^T M V, and dL/dy of the mean."""
    B = y.shape[0]
    yk = y.reshape(B, -1, y.shape[-1])[:, :, :k].astype(np.float64)
    Vb = V.reshape(B, -1, k).astype(np.float64)
    Mb = M.reshape(B, -1).astype(np.float64)
    loss = np.zeros(B)
    dy = np.zeros((B, yk.shape[1], y.shape[-1]))
    for b in range(B):
        G = yk[b].T @ (Mb[b][:, None] * yk[b])
        H = yk[b].T @ (Mb[b][:, None] * Vb[b])
        eps = 1e-6 * np.trace(G) / k + 1e-30
        C = np.linalg.solve(G + eps * np.eye(k), H)
        R = Vb[b] - yk[b] @ C
        loss[b] = np.sum(Mb[b][:, None] * R * R) / k
        dy[b, :, :k] = -2.0 * Mb[b][:, None] * (R @ C.T) / (B * k)
    return loss, dy.reshape(y.shape)
