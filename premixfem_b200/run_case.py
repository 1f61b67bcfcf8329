"""Run one setup + PCG solve on a seeded synthetic workload and print timings.

    python -m premixfem_b200.run_case --case fracture --n 128 --precision mixed

Cases (subdomains of 16^3 cells unless stated):
  fracture   n^3 fracture network (the 256^3 benchmark field at n = 256),
             p = 1 | 0 on the x faces, en_lv1 = 6, en_lv2 = 4, virtual rank
             grid (n/64)^3 with -sd 4
  grf        n^3 unit-cube GRF (sigma 2, correlation 0.1), p = 0 on x = 1,
             unit source, 8^3 subdomains, en_lv1 = 4

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
    else:
        raise SystemExit(f"unknown case {case}")
    return prob, opts


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--case", default="fracture", choices=["fracture", "grf"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--opts", default="", help="extra options appended to the generated option string")
    ap.add_argument("--learned", action="store_true", help="start the local eigensolves from the trained network")
    args = ap.parse_args()

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
