"""The solve split over processes (premixfem_b200.shard) on gloo ranks (CPU).

Each process owns a z-slab of whole virtual-rank layers.  Its local operator
and the local pieces of the oracle's three-level preconditioner (level-1
solvers of its subdomains, its part of Phi, the level-2 factors of its virtual
ranks, its level-3 V blocks and the replicated level-3 factor) stand in for
the device kernels as shard.ShardedCycle's callables; the exchanges are the
module's own: halo planes before every stencil product, the level-3 right-hand
side (and the 2-level coarse right-hand side) summed over the processes, and
the CG dots.  The assembled solution and the iteration count must match the
single-process oracle (the sums of the dot products are only reordered:
iterations +-1, solution 1e-10).
"""
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import pmf_oracle as O
from premixfem_b200 import fields, shard

CASES = {
    "grf16_w2": (2, lambda: fields.unit_cube_grf(16, seed=1), dict(sd=2, vranks=(2, 2, 2), en_lv1=4, en_lv2=3)),
    "ragged_w4": (4, lambda: fields.random_box((12, 10, 16), seed=3, sigma=1.5),
                  dict(sd=(2, 1, 1), vranks=(1, 2, 4), en_lv1=3, en_lv2=2)),
    "wcycle_w2": (2, lambda: fields.unit_cube_grf(16, seed=2),
                  dict(sd=2, vranks=(1, 2, 2), en_lv1=4, en_lv2=3, use_W_cycle=True, si_lv2=2)),
    "two_level_w2": (2, lambda: fields.unit_cube_grf(16, seed=3), dict(sd=2, vranks=(2, 1, 2), en_lv1=4, use_2level=True)),
    "neumann_null_space_w2": (2, lambda: fields.layered(seed=2, M=20, N=30, P=10, smooth_layers=4),
                              dict(sd=(2, 3, 1), vranks=(1, 1, 2), en_lv1=4, en_lv2=4, constant_null_space=True)),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _local_pieces(pc, op, slab):
    """The oracle's local mathematics on one slab, as ShardedCycle's callables."""
    lay = pc.lay
    lo, hi = slab.first_cell, slab.first_cell + slab.ncell
    elo, ehi = slab.ext_cells
    A_loc = op.A[lo:hi][:, elo:ehi].tocsr()
    subs = [i for i, s in enumerate(lay.subs) if s[6] in slab.vranks]
    d0, d1 = int(pc.dof_idx[subs[0]]), int(pc.dof_idx[subs[-1] + 1])
    Phi = pc.Phi[lo:hi][:, d0:d1].tocsr()
    nc = int(pc.dof_idx[-1])
    t, n = torch.from_numpy, lambda v: v.numpy()

    def level1(r):
        y = np.zeros(r.shape[0])
        for s in subs:
            idx = pc.sub_idx[s] - lo
            y[idx] += pc.lv1[s].solve(n(r)[idx])
        return t(y)

    def level2(c):
        z = np.zeros(c.shape[0])
        for vr in slab.vranks:
            d, f = pc.lv2[vr]
            z[d - d0] = O.chol_semidef_solve(f, n(c)[d - d0])
        return t(z)

    pieces = dict(residual=lambda x, y_ext: t(n(x) - A_loc @ n(y_ext)), level1=level1,
                  restrict=lambda r: t(Phi.T @ n(r)), prolong=lambda z: t(Phi @ n(z)), level2=level2)
    if pc.opts.use_2level:
        def coarse_rhs(c):
            cg = np.zeros(nc)
            cg[d0:d1] = n(c)
            return t(cg)

        pieces.update(coarse_rhs=coarse_rhs,
                      coarse_solve=lambda cg: t(O.chol_semidef_solve(pc.lv2c, n(cg))[d0:d1]))
    else:
        off3 = np.concatenate([[0], np.cumsum([V.shape[1] for _, V in pc.V3])])

        def level3_rhs(c):
            d3 = np.zeros(int(off3[-1]))
            for vr in slab.vranks:
                d, V = pc.V3[vr]
                d3[off3[vr]:off3[vr + 1]] = V.T @ n(c)[d - d0]
            return t(d3)

        def level3_back(w):
            z = np.zeros(d1 - d0)
            for vr in slab.vranks:
                d, V = pc.V3[vr]
                z[d - d0] = V @ n(w)[off3[vr]:off3[vr + 1]]
            return t(z)

        pieces.update(level3_rhs=level3_rhs, level3_back=level3_back,
                      level3_solve=lambda d3: t(O.chol_semidef_solve(pc.lv3, n(d3))))
    return pieces, lambda p: t(A_loc @ n(p))


def _worker(rank, world, port, name, out):
    torch.set_num_threads(1)  # several ranks share the host's cores
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        _, make, opts = CASES[name]
        prob = make()
        o = O.Options(**opts)
        op = O.Operator(prob)
        pc = O.Preconditioner(op, o)
        slab = shard.plan_slabs(prob["mesh"], o.vranks, world)[rank]
        halo = shard.Halo(slab)
        pieces, stencil = _local_pieces(pc, op, slab)
        cycle = shard.ShardedCycle(pc.schedule(), halo, **pieces)

        def matvec(p):
            return stencil(halo.extend(p))

        b = op.rhs()
        lo, hi = slab.first_cell, slab.first_cell + slab.ncell
        x, its, hist, reason = shard.pcg(torch.from_numpy(b[lo:hi].copy()), matvec, cycle.apply, op.n,
                                         rtol=pc.opts.rtol, null_space=o.constant_null_space)
        xg = torch.zeros(op.n, dtype=torch.float64)
        xg[lo:hi] = x
        dist.all_reduce(xg)
        if rank == 0:
            np.save(out, xg.numpy())
            with open(out + ".txt", "w") as f:
                f.write(f"{its} {reason} {halo.exchanges} {cycle.sums}\n")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", sorted(CASES))
def test_sharded_solve_matches_single_process(name, tmp_path, monkeypatch):
    world, make, opts = CASES[name]
    out = str(tmp_path / "x.npy")
    # one BLAS / OpenMP thread per rank (read when the spawned ranks import numpy)
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        monkeypatch.setenv(v, "1")
    mp.spawn(_worker, args=(world, _free_port(), name, out), nprocs=world, join=True)
    x = np.load(out)
    its, reason, exchanges, sums = open(out + ".txt").read().split()
    prob = make()
    ref = O.solve(prob, O.Options(**opts))
    assert reason == ref["reason"] == "converged_rtol"
    assert abs(int(its) - ref["its"]) <= 1, (its, ref["its"])
    a, b = ref["x"], x
    if not prob["dirichlet"]:
        a, b = a - a.mean(), b - b.mean()
    assert np.linalg.norm(b - a) <= 1e-10 * np.linalg.norm(a)
    # one halo exchange per A p of the CG step and per residual of the cycle
    # after its first visit: its preconditioner applications and its A p
    sched = ref["pc"].schedule()
    assert int(exchanges) == int(its) * len(sched)
    # one coarse right-hand side summed per level-3 (or 2-level) visit of each application
    assert int(sums) == int(its) * sum(1 for lvl in sched if lvl in (3, "2g"))


def test_slab_plan():
    slabs = shard.plan_slabs((12, 10, 17), (2, 1, 4), 2)
    assert [(s.z0, s.z1) for s in slabs] == [(0, 9), (9, 17)]  # z-layers 5, 4, 4, 4
    assert slabs[0].vranks == [0, 1, 2, 3] and slabs[1].vranks == [4, 5, 6, 7]
    assert slabs[0].below is None and slabs[0].above == 1 and slabs[1].below == 0 and slabs[1].above is None
    assert slabs[0].ext_cells == (0, 10 * 120) and slabs[1].ext_cells == (8 * 120, 17 * 120)
    with pytest.raises(ValueError):
        shard.plan_slabs((12, 10, 17), (2, 1, 3), 2)
