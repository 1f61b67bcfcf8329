"""The solve split over processes (premixfem_b200.shard) on gloo ranks (CPU).

Each process owns a z-slab of whole virtual-rank layers and sets up its part
of the oracle's three-level preconditioner from its slab and the two ghost
planes around it only: the level-1 solvers of its subdomains, their local
bases, the level-2 factors of its virtual ranks and their level-3 vectors.
The one set-up exchange is the module's own: the basis (Psi, or Phi for the
2-level branch) on the two boundary planes to the neighbours, from which each
process adds its coupling to the slab above to the global coarse matrix, and
one all-reduce of that matrix and of the per-rank coarse counts.  These
pieces stand in for the device kernels as shard.ShardedCycle's callables; the
solve's exchanges are the module's too: halo planes before every stencil
product, the level-3 right-hand side (and the 2-level coarse right-hand side)
summed over the processes, and the CG dots (in PETSc's order, and fused: p.w,
then ||r||^2 and z.r in one sum; the counts of each are checked).  The
assembled solution and the iteration count must match the single-process
oracle (sums and products are only reordered: iterations +-1, solution
1e-10).
"""
import socket

import numpy as np
import pytest
import scipy.sparse as sp
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


def _sharded_setup(prob, o, slab, slabs):
    """This process's part of the three-level preconditioner, built from its
    slab and the two ghost planes around it only (the problem cropped to
    planes z0 - 1 .. z1), with the set-up exchanges of premixfem_b200.shard:
    the basis on the boundary planes to the neighbours, the coarse counts and
    the global coarse matrix summed over the processes.  Returns
    ShardedCycle's callables, the local stencil product on halo-extended
    vectors, this slab's right-hand side and the set-up's exchange count."""
    M, N, P = prob["mesh"]
    mn = M * N
    lay = O.Layout.build(prob["mesh"], o.vranks, o.sd)
    crop, cbox = O.crop_around(prob, (0, M, 0, N, slab.z0, slab.z1 - slab.z0))
    opc = O.Operator(crop)
    zc = slab.z0 - cbox[4]  # first crop plane in global z
    off, nloc = cbox[4] * mn, slab.ncell  # the slab's cells in the crop's numbering
    rows = slice(off, off + nloc)
    t, n = torch.from_numpy, lambda v: v.numpy()

    def to_crop(box):
        return (box[0], box[1], box[2], box[3], box[4] - zc, box[5]) + tuple(box[6:])

    # level 1 and the local bases: subdomain by subdomain, from the crop alone
    subs = [s_ for s_ in lay.subs if s_[6] in slab.vranks]
    sub_idx, lv1, phi, nums = [], [], [], []
    for s_ in subs:
        bc = to_crop(s_)
        sub_idx.append(O.box_cells(crop["mesh"], bc) - off)
        Aloc = opc.principal(bc)
        lv1.append(O.CholSolver(Aloc) if o.use_full_Cholesky_lv1 else O.IC0Solver(Aloc))
        w, V, num, _ = O.local_basis(opc, bc, o)
        phi.append(V)
        nums.append(num)
    dof = np.concatenate([[0], np.cumsum(nums)]).astype(int)
    nd = int(dof[-1])
    Phi = sp.csr_matrix((np.concatenate([phi[i][:, j] for i in range(len(subs)) for j in range(nums[i])]),
                         (np.concatenate([sub_idx[i] for i in range(len(subs)) for j in range(nums[i])]),
                          np.concatenate([np.full(sub_idx[i].size, dof[i] + j)
                                          for i in range(len(subs)) for j in range(nums[i])]))),
                        shape=(nloc, nd))
    A_slab = opc.A[rows][:, rows].tocsr()
    A2 = (Phi.T @ A_slab @ Phi).toarray()
    spr = lay.subs_per_rank
    rdof = {r: np.arange(dof[i * spr], dof[(i + 1) * spr]) for i, r in enumerate(slab.vranks)}
    lv2 = {r: O.chol_semidef(A2[np.ix_(d, d)]) for r, d in rdof.items()}
    # the faces between the top plane and the ghost plane above: tz of the ghost plane's cells
    t_up = opc.tz[slab.z1 - zc].ravel() if slab.above is not None else None
    exchanges = 0

    def coarse(basis, counts_mine):
        """The global coarse matrix basis^T A basis from this slab's block and
        its coupling to the slab above (the neighbours' basis on the facing
        planes arrives by exchange_planes)."""
        nonlocal exchanges
        counts = shard.coarse_counts(len(lay.ranks), counts_mine)
        offs = np.concatenate([[0], np.cumsum(counts)]).astype(int)
        lo_, hi_ = offs[slab.vranks[0]], offs[slab.vranks[-1] + 1]
        m = np.zeros((offs[-1], offs[-1]))
        m[lo_:hi_, lo_:hi_] = basis.T @ (A_slab @ basis)
        bt = torch.from_numpy(np.ascontiguousarray(basis[nloc - mn:]))
        bb = torch.from_numpy(np.ascontiguousarray(basis[:mn]))
        _, from_above = shard.exchange_planes(slab, bt, bb)
        exchanges += 1
        if from_above is not None:
            up = slabs[slab.rank + 1].vranks
            ua, ub = offs[up[0]], offs[up[-1] + 1]
            cpl = basis[nloc - mn:].T @ (-t_up[:, None] * from_above.numpy())
            m[lo_:hi_, ua:ub] += cpl
            m[ua:ub, lo_:hi_] += cpl.T
        mt = shard.sum_coarse(torch.from_numpy(m))
        return mt.numpy(), offs, lo_, hi_

    def level1(r):
        y = np.zeros(r.shape[0])
        for idx, sol in zip(sub_idx, lv1):
            y[idx] += sol.solve(n(r)[idx])
        return t(y)

    def level2(c):
        z = np.zeros(c.shape[0])
        for r, d in rdof.items():
            z[d] = O.chol_semidef_solve(lv2[r], n(c)[d])
        return t(z)

    pieces = dict(level1=level1, restrict=lambda r: t(Phi.T @ n(r)), prolong=lambda z: t(Phi @ n(z)),
                  level2=level2)
    if o.use_2level:
        Ac, offs, lo_, hi_ = coarse(Phi.toarray(), {r: d.size for r, d in rdof.items()})
        if not o.no_shift_A_cc:
            Ac = Ac + O.NIL * np.eye(Ac.shape[0])
        fac = O.chol_semidef(Ac)

        def coarse_rhs(c):
            cg = np.zeros(Ac.shape[0])
            cg[lo_:hi_] = n(c)
            return t(cg)

        pieces.update(coarse_rhs=coarse_rhs, coarse_solve=lambda cg: t(O.chol_semidef_solve(fac, n(cg))[lo_:hi_]))
    else:
        V3 = {}
        for r, d in rdof.items():
            bc = to_crop(lay.ranks[r])
            cells = O.box_cells(crop["mesh"], bc) - off
            PhiR = Phi[cells][:, d]
            V3[r] = O.level3_basis(PhiR.T @ opc.neumann(bc) @ PhiR, o)[1]
        Vloc = np.zeros((nd, sum(V.shape[1] for V in V3.values())))
        c0 = 0
        for r, d in rdof.items():
            Vloc[d, c0:c0 + V3[r].shape[1]] = V3[r]
            c0 += V3[r].shape[1]
        Psi = np.asarray(Phi @ Vloc)
        A3, off3, lo_, hi_ = coarse(Psi, {r: V.shape[1] for r, V in V3.items()})
        if not o.no_shift_A_cc:
            A3 = A3 + O.NIL * np.eye(A3.shape[0])  # :1361-1363
        fac = O.chol_semidef(A3)

        def level3_rhs(c):
            d3 = np.zeros(A3.shape[0])
            d3[lo_:hi_] = Vloc.T @ n(c)
            return t(d3)

        pieces.update(level3_rhs=level3_rhs, level3_back=lambda w: t(Vloc @ n(w)[lo_:hi_]),
                      level3_solve=lambda d3: t(O.chol_semidef_solve(fac, n(d3))))
    A_loc = opc.A[rows].tocsr()  # slab rows, crop columns: [ghost below | slab | ghost above]
    pieces["residual"] = lambda x, y_ext: t(n(x) - A_loc @ n(y_ext))
    b = np.asarray(prob["source"])[slab.z0:slab.z1].ravel() + opc.bval.ravel()[rows]
    return pieces, (lambda p_: t(A_loc @ n(p_))), b, exchanges


def _worker(rank, world, port, name, fused, out):
    torch.set_num_threads(1)  # several ranks share the host's cores
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        _, make, opts = CASES[name]
        prob = make()
        o = O.Options(**opts).normalized()
        slabs = shard.plan_slabs(prob["mesh"], o.vranks, world)
        slab = slabs[rank]
        halo = shard.Halo(slab)
        pieces, stencil, b, setup_exchanges = _sharded_setup(prob, o, slab, slabs)
        cycle = shard.ShardedCycle(O.cycle_schedule(o), halo, **pieces)

        def matvec(p):
            return stencil(halo.extend(p))

        n_global = int(np.prod(prob["mesh"]))
        stats = {}
        x, its, hist, reason = shard.pcg(torch.from_numpy(b), matvec, cycle.apply, n_global,
                                         rtol=o.rtol, null_space=o.constant_null_space, fused=fused, stats=stats)
        xg = torch.zeros(n_global, dtype=torch.float64)
        lo, hi = slab.first_cell, slab.first_cell + slab.ncell
        xg[lo:hi] = x
        dist.all_reduce(xg)
        if rank == 0:
            np.save(out, xg.numpy())
            with open(out + ".txt", "w") as f:
                f.write(f"{its} {reason} {halo.exchanges} {cycle.sums} {setup_exchanges} {stats['allreduces']} "
                        f"{stats['pc_applications']}\n")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,fused", [(n, False) for n in sorted(CASES)]
                         + [("grf16_w2", True), ("neumann_null_space_w2", True), ("two_level_w2", True)])
def test_sharded_solve_matches_single_process(name, fused, tmp_path, monkeypatch):
    world, make, opts = CASES[name]
    out = str(tmp_path / "x.npy")
    # one BLAS / OpenMP thread per rank (read when the spawned ranks import numpy)
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        monkeypatch.setenv(v, "1")
    mp.spawn(_worker, args=(world, _free_port(), name, fused, out), nprocs=world, join=True)
    x = np.load(out)
    its, reason, exchanges, sums, setup_exchanges, allreduces, napply = (
        int(v) if v.isdigit() else v for v in open(out + ".txt").read().split())
    prob = make()
    ref = O.solve(prob, O.Options(**opts))
    assert reason == ref["reason"] == "converged_rtol"
    assert abs(its - ref["its"]) <= 1, (its, ref["its"])
    a, b = ref["x"], x
    if not prob["dirichlet"]:
        a, b = a - a.mean(), b - b.mean()
    assert np.linalg.norm(b - a) <= 1e-10 * np.linalg.norm(a)
    # preconditioner applications: PETSc's order one per iteration (the first
    # before the loop, none after the converging residual); the fused form one more
    assert napply == its + (1 if fused else 0)
    # scalar all-reduces: p.w per iteration, then PETSc's order ||r||^2 and z.r
    # separately (and sum z with the null space), the fused form all in one
    null = 1 if opts.get("constant_null_space") else 0
    assert allreduces == (2 * its + 1 if fused else 3 * its + 1 + null * its), allreduces
    # one halo exchange per A p of the CG step and per residual of the cycle
    # after its first visit
    sched = ref["pc"].schedule()
    assert exchanges == its + napply * (len(sched) - 1)
    # one coarse right-hand side summed per level-3 (or 2-level) visit of each application
    assert sums == napply * sum(1 for lvl in sched if lvl in (3, "2g"))
    # the set-up exchanged the basis on the boundary planes once (Psi, or Phi for the 2-level branch)
    assert setup_exchanges == 1


def test_slab_plan():
    slabs = shard.plan_slabs((12, 10, 17), (2, 1, 4), 2)
    assert [(s.z0, s.z1) for s in slabs] == [(0, 9), (9, 17)]  # z-layers 5, 4, 4, 4
    assert slabs[0].vranks == [0, 1, 2, 3] and slabs[1].vranks == [4, 5, 6, 7]
    assert slabs[0].below is None and slabs[0].above == 1 and slabs[1].below == 0 and slabs[1].above is None
    assert slabs[0].ext_cells == (0, 10 * 120) and slabs[1].ext_cells == (8 * 120, 17 * 120)
    with pytest.raises(ValueError):
        shard.plan_slabs((12, 10, 17), (2, 1, 3), 2)


def test_exchange_planes_takes_cell_by_column_tensors():
    # the shape check comes before any communication
    slab = shard.plan_slabs((4, 4, 8), (1, 1, 2), 2)[0]
    with pytest.raises(ValueError):
        shard.exchange_planes(slab, torch.zeros(16), torch.zeros(16))
