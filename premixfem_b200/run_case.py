"""Run one setup + PCG solve on a seeded synthetic workload and print timings.

    python -m premixfem_b200.run_case --case fracture --n 128 --precision mixed

Cases (subdomains of 16^3 cells unless stated):
  fracture   n^3 fracture network (the 256^3 benchmark field at n = 256),
             p = 1 | 0 on the x faces, en_lv1 = 6, en_lv2 = 4, virtual rank
             grid (n/64)^3 with -sd 4
  grf        n^3 unit-cube GRF (sigma 2, correlation 0.1), p = 0 on x = 1,
             unit source, 8^3 subdomains, en_lv1 = 4
  layered    60 x 220 x 85 layered channel field (cells 20 x 10 x 2, channel
             contrast 1e6, +/-1 injector/producer, pure Neumann): 6 x 22 x 17
             subdomains of 10 x 10 x 5 on a 2 x 2 x 1 virtual rank grid (the
             per-rank dense coarse inverse holds at most 4096 unknowns),
             en_lv1 = 4, -ksp_constant_null_space; --n is ignored
  large      n x n x n/2 anisotropic GRF (sigma 3) with fracture planes of
             contrast 1e6, p = 0 on z = 0 (512 x 512 x 256 at n = 512):
             16^3 subdomains, -sd 4 on an (n/64, n/64, n/128) virtual rank
             grid (64 subdomains, 512 coarse unknowns per rank), en_lv1 = 8,
             en_lv2 = 4
  batch      --count independent unit-cube GRF problems (per-axis sizes
             U{24..80}, sigma U[1,3], correlation U[0.05,0.2], p = 0 on
             x = 1), ~8^3 ragged subdomains, en_lv1 = 4; one set-up and four
             right-hand sides (unit + 3 N(0,1)) each; --n is ignored

This is the driver the kernel profiles are taken on (a small case of the
benchmark's kernels under a profiler), and a quick way to try options:
--opts passes extra PETSc-style options, e.g. "-use_W_cycle -si_lv1 2".
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from premixfem_b200 import fields
from premixfem_b200.solver import DarcySolver, options_string


def make_case(case, n, seed):
    if case == "fracture":
        if n % 64:
            raise SystemExit("--n must be a multiple of 64 for the fracture case")
        prob = fields.fracture256(n, seed=seed)
        v = n // 64
        opts = {"sd": 4, "pmf_vranks": (v, v, v), "en_lv1": 6, "en_lv2": 4}
    elif case == "grf":
        if n % 8:
            raise SystemExit("--n must be a multiple of 8 for the grf case")
        prob = fields.unit_cube_grf(n, seed=seed)
        opts = {"sd": n // 8, "en_lv1": 4, "en_lv2": 4}
    elif case == "layered":
        prob = fields.layered(seed=seed)
        opts = {"pmf_sd": (3, 11, 17), "pmf_vranks": (2, 2, 1), "en_lv1": 4, "en_lv2": 4,
                "ksp_constant_null_space": True}
    elif case == "large":
        if n % 256:
            raise SystemExit("--n must be a multiple of 256 for the large case")
        f = n / 512.0
        prob = fields.large_frac(M=n, N=n, P=n // 2, seed=seed, n_frac=max(1, int(400 * f * f)),
                                 frac_lo=max(4, int(32 * f)), frac_hi=int(256 * f))
        opts = {"sd": 4, "pmf_vranks": (n // 64, n // 64, n // 128), "en_lv1": 8, "en_lv2": 4}
    else:
        raise SystemExit(f"unknown case {case}")
    return prob, opts


def run_batch(args):
    """The batching workload through one BatchSolver: one batched set-up (every
    phase one launch over all problems' subdomains) and four batched solves
    (one CG per problem); per problem the iteration counts, then the totals."""
    import torch

    from premixfem_b200.solver import BatchSolver

    batch = fields.grf_batch(count=args.count, seed=args.seed)
    problems = [p for p, _ in batch]
    s = BatchSolver(problems, [fields.tiles(p["mesh"]) for p in problems],
                    options_string({"en_lv1": 4, "en_lv2": 4, "pmf_precision": args.precision}) + " " + args.opts)
    for rep in range(args.repeat):
        s.set_kappa_problems(problems)
        s.setup()
        su, _ = s.timing()
        its_all, solve_ms = [], 0.0
        for j in range(4):
            b = s.rhs(torch.from_numpy(s.pack([srcs[j] for _, srcs in batch])).cuda())
            x = torch.empty_like(b)
            _, its, _, reasons = s.solve(b, x)
            bad = [q for q, r in enumerate(reasons) if r != "converged"]
            if bad:
                raise SystemExit(f"right-hand side {j}: problems {bad} did not converge ({reasons[bad[0]]})")
            its_all.append([int(v) for v in its])
            solve_ms += s.timing()[1]
        print(json.dumps({"case": "batch", "problems": args.count, "rhs": 4 * args.count, "precision": args.precision,
                          "rep": rep, "setup_ms": round(su, 3), "solve_ms": round(solve_ms, 3),
                          "stages_ms": {k: round(v, 3) for k, v in s.stages().items()},
                          "pcg_iters_mean": float(np.mean(its_all)), "pcg_iters_max": int(np.max(its_all)),
                          "pcg_iters_per_problem": [list(v) for v in zip(*its_all)]}), flush=True)
    s.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--case", default="fracture", choices=["fracture", "grf", "layered", "large", "batch"])
    ap.add_argument("--count", type=int, default=64, help="problems of the batch case")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--opts", default="", help="extra options appended to the generated option string")
    ap.add_argument("--learned", action="store_true", help="start the local eigensolves from the trained network")
    args = ap.parse_args()

    if args.case == "batch":
        run_batch(args)
        return
    import torch

    prob, opts = make_case(args.case, args.n, args.seed)
    if args.learned:
        from premixfem_b200.learned import DEFAULT_WEIGHTS
        opts["pmf_learned"] = DEFAULT_WEIGHTS
    o = options_string(dict(opts, pmf_precision=args.precision)) + " " + args.opts
    s = DarcySolver(prob["dom"], prob["mesh"], o)
    for f, v in prob["dirichlet"].items():
        s.set_dirichlet(f, v)
    kx = torch.from_numpy(np.ascontiguousarray(prob["kappa"][0]).ravel()).cuda()
    ky = torch.from_numpy(np.ascontiguousarray(prob["kappa"][1]).ravel()).cuda()
    kz = torch.from_numpy(np.ascontiguousarray(prob["kappa"][2]).ravel()).cuda()
    src = torch.from_numpy(np.ascontiguousarray(prob["source"]).ravel()).cuda()
    for rep in range(args.repeat):
        s.set_kappa(kx, ky, kz)
        s.setup()
        b = torch.empty_like(src)
        s.rhs(src, b)
        x = torch.empty_like(src)
        _, its, rn, reason = s.solve(b, x)
        su, so = s.timing()
        _, _, it1, st1 = s.eigen_lv1()
        _, _, it3 = s.eigen_lv2()
        stages = {k_: round(v_ * 1e3, 2) for k_, v_ in s.stages().items()}
        print(json.dumps({"case": args.case, "n": args.n, "precision": args.precision, "rep": rep,
                          "setup_ms": round(su, 3), "solve_ms": round(so, 3), "pcg_iters": its,
                          "stages_ms_cumulative": stages,
                          "reason": reason, "eig_iters_mean": float(it1.mean()), "eig_iters_max": int(it1.max()),
                          "eig_not_converged": int((st1 == 1).sum()), "lv3_iters_max": int(it3.max()),
                          "lv3_iters_mean": float(it3.mean())}), flush=True)
    s.close()


if __name__ == "__main__":
    main()
