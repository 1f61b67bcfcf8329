"""Learned initial blocks for the local eigensolves: training and evaluation.

    python -m premixfem_b200.learned train --out premixfem_b200/weights/fracture16_k6.pmfnet
    python -m premixfem_b200.learned eval --weights premixfem_b200/weights/fracture16_k6.pmfnet --n 128

Training data come from the method's own set-up: for each seeded field of the
256^3 fracture distribution the solver runs its plain (randomly started)
batched eigensolve, and `pmf_learned_patches` returns, per 16^3 subdomain,
the network input (log-permeability patch, Dirichlet and inside masks), the
k converged local eigenvectors and the mass diagonal of the eigenproblem.
The network (pmf_net.h: 3-D conv encoder-decoder, 0.53 M parameters, BF16
weights) is trained with the library's own forward, backward and Adam
kernels on the subspace loss ||V - Y C||_M^2 / k, C = (Y^T M Y)^-1 Y^T M V,
which does not care about the order, sign or mixing of the k vectors -- only
their span, which is what LOBPCG's first Rayleigh-Ritz step uses.

torch only allocates device memory here; every computation is a library
kernel called through the C ABI.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from premixfem_b200 import _native, fields
from premixfem_b200.solver import DarcySolver, options_string

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "fracture16_k6.pmfnet")
VOX = 4096
CH = 16


def _p(t):
    return C.c_void_p(t.data_ptr())


class Net:
    """The library's network object (pmf_net) with device tensors from torch."""

    def __init__(self, seed=1, path=None):
        self.lib = _native.load()
        h = C.c_void_p()
        if path:
            _native.check(self.lib.pmf_net_load(path.encode(), C.byref(h)))
        else:
            _native.check(self.lib.pmf_net_create(C.c_ulonglong(seed), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.pmf_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        return int(self.lib.pmf_net_params(self.h))

    @staticmethod
    def layers():
        lib = _native.load()
        out = []
        for l in range(9):
            info = (C.c_int * 6)()
            _native.check(lib.pmf_net_layer_info(l, info))
            out.append(tuple(info))
        return out

    def forward(self, x, y):
        _native.check(self.lib.pmf_net_forward(self.h, _p(x), int(x.shape[0]), _p(y)))

    def backward(self, dy):
        _native.check(self.lib.pmf_net_backward(self.h, _p(dy), int(dy.shape[0])))

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        _native.check(self.lib.pmf_net_adam(self.h, C.c_float(lr), C.c_float(b1), C.c_float(b2), C.c_float(eps),
                                            C.c_float(wd)))

    def save(self, path):
        _native.check(self.lib.pmf_net_save(self.h, path.encode()))

    def weights(self, layer):
        typ, cin, cout, si, so, taps = self.layers()[layer]
        w = np.zeros((taps, cin, cout), dtype=np.float32)
        b = np.zeros(cout, dtype=np.float32)
        _native.check(self.lib.pmf_net_get_weights(self.h, layer, w.ctypes.data_as(C.c_void_p),
                                                   b.ctypes.data_as(C.c_void_p)))
        return w, b

    def set_weights(self, layer, w, b):
        w = np.ascontiguousarray(w, dtype=np.float32)
        b = np.ascontiguousarray(b, dtype=np.float32)
        _native.check(self.lib.pmf_net_set_weights(self.h, layer, w.ctypes.data_as(C.c_void_p),
                                                   b.ctypes.data_as(C.c_void_p)))

    def grads(self, layer):
        typ, cin, cout, si, so, taps = self.layers()[layer]
        w = np.zeros((taps, cin, cout), dtype=np.float32)
        b = np.zeros(cout, dtype=np.float32)
        _native.check(self.lib.pmf_net_get_grads(self.h, layer, w.ctypes.data_as(C.c_void_p),
                                                 b.ctypes.data_as(C.c_void_p)))
        return w, b


def loss_and_grad(y, V, M, k, loss, dy):
    lib = _native.load()
    _native.check(lib.pmf_net_loss(_p(y), _p(V), _p(M), int(y.shape[0]), int(k), _p(loss), _p(dy)))


def fracture_solver(n, seed, precision="mixed", learned=None, extra=None):
    prob = fields.fracture256(n, seed=seed)
    v = n // 64
    opts = {"sd": 4, "pmf_vranks": (v, v, v), "en_lv1": 6, "en_lv2": 4, "pmf_precision": precision}
    if learned:
        opts["pmf_learned"] = learned
    opts.update(extra or {})
    s = DarcySolver(prob["dom"], prob["mesh"], options_string(opts))
    for f, val in prob["dirichlet"].items():
        s.set_dirichlet(f, val)
    return prob, s


def patches(n, seed, precision="mixed"):
    """(feats BF16, V, M) device tensors for every subdomain of one seeded fracture field."""
    import torch
    prob, s = fracture_solver(n, seed, precision)
    k = [torch.from_numpy(np.ascontiguousarray(kk).ravel()).cuda() for kk in prob["kappa"]]
    s.set_kappa(*k)
    s.setup()
    nsub = s.info()["nsub"]
    feats = torch.empty((nsub, VOX, CH), dtype=torch.bfloat16, device="cuda")
    V = torch.empty((nsub, VOX, 6), dtype=torch.float32, device="cuda")
    M = torch.empty((nsub, VOX), dtype=torch.float32, device="cuda")
    _native.check(s.lib.pmf_learned_patches(s.h, _p(feats), _p(V), _p(M)))
    s.close()
    return feats, V, M


def augment(xb, Vb, Mb, sym):
    """Apply one of the 8 exact symmetries of the local eigenproblem to a batch of full 16^3 patches.

    Flips along y and z and the y<->z exchange map a subdomain's eigenproblem onto
    another valid one (the mass matrix treats y and z alike; x is not symmetric:
    the reference's x-face accumulation is one-sided).  Bit 0: flip y, bit 1: flip z,
    bit 2: exchange y and z (with the y and z permeability channels).
    """
    import torch
    B = xb.shape[0]
    x = xb.view(B, 16, 16, 16, -1)
    v = Vb.view(B, 16, 16, 16, -1)
    m = Mb.view(B, 16, 16, 16)
    if sym & 1:
        x, v, m = x.flip(2), v.flip(2), m.flip(2)
    if sym & 2:
        x, v, m = x.flip(1), v.flip(1), m.flip(1)
    if sym & 4:
        x, v, m = x.transpose(1, 2), v.transpose(1, 2), m.transpose(1, 2)
        x = x[..., torch.tensor([0, 2, 1] + list(range(3, x.shape[-1])), device=x.device)]
    return (x.reshape(B, VOX, -1).contiguous(), v.reshape(B, VOX, -1).contiguous(), m.reshape(B, VOX).contiguous())


def train(out, seeds, val_seed, n=256, epochs=20, batch=64, lr=2e-3, seed=1, log=print):
    import torch
    t0 = time.time()
    data = [patches(n, sd) for sd in seeds]
    feats = torch.cat([d[0] for d in data])
    V = torch.cat([d[1] for d in data])
    M = torch.cat([d[2] for d in data])
    del data
    vf, vV, vM = patches(n, val_seed)
    nval = min(1024, vf.shape[0])
    vf, vV, vM = vf[:nval].contiguous(), vV[:nval].contiguous(), vM[:nval].contiguous()
    log(f"data: {feats.shape[0]} training patches, {nval} validation patches, {time.time() - t0:.1f} s")
    net = Net(seed=seed)
    N = feats.shape[0]
    steps_per_epoch = N // batch
    total = epochs * steps_per_epoch
    y = torch.empty((batch, VOX, CH), dtype=torch.float32, device="cuda")
    dy = torch.empty_like(y)
    loss = torch.empty(batch, dtype=torch.float32, device="cuda")
    g = torch.Generator(device="cpu").manual_seed(seed)

    def validate():
        ls = []
        yv = torch.empty((batch, VOX, CH), dtype=torch.float32, device="cuda")
        dv = torch.empty_like(yv)
        lv = torch.empty(batch, dtype=torch.float32, device="cuda")
        for i in range(0, nval - batch + 1, batch):
            net.forward(vf[i:i + batch], yv)
            loss_and_grad(yv, vV[i:i + batch], vM[i:i + batch], 6, lv, dv)
            ls.append(lv.clone())
        return float(torch.cat(ls).mean())

    hist = []
    step = 0
    t1 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(N, generator=g).cuda()
        run = 0.0
        for it in range(steps_per_epoch):
            idx = perm[it * batch:(it + 1) * batch]
            xb, Vb, Mb = augment(feats[idx], V[idx], M[idx], int(torch.randint(0, 8, (1,), generator=g)))
            net.forward(xb, y)
            loss_and_grad(y, Vb, Mb, 6, loss, dy)
            net.backward(dy)
            cur = lr * 0.5 * (1.0 + math.cos(math.pi * step / total))
            net.adam(cur, wd=1e-5)
            run += float(loss.mean())
            step += 1
        val = validate()
        hist.append({"epoch": ep, "train_loss": run / steps_per_epoch, "val_loss": val,
                     "seconds": round(time.time() - t1, 1)})
        log(json.dumps(hist[-1]))
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    net.save(out)
    return hist


def evaluate(weights, n=128, seed=77, precision="mixed", learned_its=60, eig_tol=None):
    """Set-up and solve with and without the learned start on one held-out field."""
    import torch
    res = {}
    for mode in ("random", "learned"):
        extra = {"pmf_learned_its": learned_its} if mode == "learned" else {}
        if eig_tol:
            extra["pmf_eig_tol"] = eig_tol
        prob, s = fracture_solver(n, seed, precision, learned=weights if mode == "learned" else None, extra=extra)
        k = [torch.from_numpy(np.ascontiguousarray(kk).ravel()).cuda() for kk in prob["kappa"]]
        src = torch.from_numpy(np.ascontiguousarray(prob["source"]).ravel()).cuda()
        for _ in range(2):  # second run is timed warm
            s.set_kappa(*k)
            s.setup()
            b = torch.empty_like(src)
            s.rhs(src, b)
            x = torch.empty_like(src)
            _, its, rn, reason = s.solve(b, x)
        su, so = s.timing()
        _, _, it1, st1 = s.eigen_lv1()
        st = (C.c_longlong * 4)()
        nm = C.c_double()
        _native.check(s.lib.pmf_get_learned_stats(s.h, st, C.byref(nm)))
        res[mode] = {"setup_ms": su, "solve_ms": so, "pcg_iters": its, "eig_iters_mean": float(it1.mean()),
                     "eig_iters_max": int(it1.max()), "fallbacks": int(st[1]), "net_ms": nm.value,
                     "x": x.cpu().numpy()}
        s.close()
    xr, xl = res["random"].pop("x"), res["learned"].pop("x")
    res["solution_rel_diff"] = float(np.linalg.norm(xl - xr) / np.linalg.norm(xr))
    return res


def time_forward(weights, batch, reps):
    """Forward passes of the network on `batch` random 16^3 patches: ms per pass
    (CUDA events after one untimed pass)."""
    import torch

    net = Net(path=weights)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((batch, 4096, 16), device="cuda", generator=g).to(torch.bfloat16)
    y = torch.empty((batch, 4096, 16), dtype=torch.float32, device="cuda")
    net.forward(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.forward(x, y)
    e1.record()
    torch.cuda.synchronize()
    net.close()
    return {"batch": batch, "reps": reps, "ms_per_forward": e0.elapsed_time(e1) / reps}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--seeds", default="101,102,103,104,105,106,107,108,109,110")
    t.add_argument("--val-seed", type=int, default=111)
    t.add_argument("--n", type=int, default=256)
    t.add_argument("--epochs", type=int, default=30)
    t.add_argument("--batch", type=int, default=64)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--log", default=None)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=DEFAULT_WEIGHTS)
    e.add_argument("--n", type=int, default=128)
    e.add_argument("--seed", type=int, default=77)
    e.add_argument("--precision", default="mixed")
    e.add_argument("--learned-its", type=int, default=60)
    e.add_argument("--eig-tol", type=float, default=None)
    f = sub.add_parser("forward", help="time the forward pass on random patches (CUDA events)")
    f.add_argument("--weights", default=DEFAULT_WEIGHTS)
    f.add_argument("--batch", type=int, default=512)
    f.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    if a.cmd == "forward":
        print(json.dumps(time_forward(a.weights, a.batch, a.reps)))
        return
    if a.cmd == "train":
        fh = open(a.log, "w") if a.log else None

        def log(msg):
            print(msg, flush=True)
            if fh:
                fh.write(msg + "\n")
                fh.flush()
        train(a.out, [int(x) for x in a.seeds.split(",")], a.val_seed, a.n, a.epochs, a.batch, a.lr, log=log)
    else:
        print(json.dumps(evaluate(a.weights, a.n, a.seed, a.precision, a.learned_its, a.eig_tol)))


if __name__ == "__main__":
    main()
