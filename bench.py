#!/usr/bin/env python
"""Benchmark: setup + preconditioned CG solve of the three-level GMsFEM
preconditioner on one B200 (per rank), through libpremixfem_b200.so.

Metric: setup+solve seconds at 1e-8 relative residual and PCG iterations,
mixed precision with the learned eigensolver start (FP32 preconditioner and
eigensolver vectors, FP64 PCG, Rayleigh-Ritz and coarse factorisations;
local eigensolves started from the trained network's blocks, Ritz-gated,
random restart on failure) against the plain FP64 GPU form.

One step = one full setup (operator assembly, level-1 IC(0), batched local
eigensolves, Galerkin level 2, level-3 eigensolve + Galerkin, coarse
inverses) plus one PCG solve to 1e-8 on the workload's seeded synthetic field.

Forms measured on the headline workload (fracture256):
  value        mixed form with the learned start, inputs resident in HBM
  mixed_nonet  the mixed form with random eigensolver starts (the network's own gain)
  plain_fp64   plain FP64 form (random starts), the comparator the metric names
  e2e          the mixed/learned form through the C ABI with host buffers
               (host->device copies of kappa and source, device->host copies
               of the right-hand side and solution, inside the timed region)
Accuracy: every form's solution against an FP64 reference solution (the
device FP64 form solved to relative residual 1e-13; 1e-10 and modulo
constants for the pure-Neumann layered field), true residuals, the
local eigensolvers' stop codes; in the CPU-baseline leg, a seeded sample of
64 subdomains' local eigenvalues against the oracle's exact local GHEPs.
Roofline: the kernels of one PCG iteration timed by class with CUDA events
on the solver stream (pmf_profile_iteration); the dominant class is the
`roofline` object.

Secondary workloads (--extra, default "fracture256_2level,layered,large512,
batch64") run after the headline with their own 3 warm-up + 3 timed steps per
form and are reported under "workloads" in the same line; they and the CPU
baseline run at N = 1 only.

Multi-GPU (torchrun, N ranks): every rank solves its own seeded replica on
its own GPU (no data-path collective: replicas only); step time is the max
over ranks.

--impl reference times the reference algorithm's CPU restatement (the C++/OpenMP
port under oracle/cpu_ref, FP64, all host threads; the reference itself needs
PETSc/SLEPc/MPI and cannot be built here) on the same
workload: each timed step is the full 256^3 solve (about 35 s on 16 host
cores); warm-up steps run a 128^3 crop.
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from premixfem_b200 import fields  # noqa: E402
from premixfem_b200.solver import options_string  # noqa: E402

METRIC = "setup+solve s at 1e-8 resid & PCG iters: mixed/learned vs plain FP64, 1 B200"

WORKLOADS = {
    # 256^3 fracture network, 16^3 subdomains of 16^3 cells, k = 6 (the benchmarked workload).
    "fracture256": dict(
        make=lambda seed: fields.fracture256(256, seed=seed),
        opts={"sd": 4, "pmf_vranks": (4, 4, 4), "en_lv1": 6, "en_lv2": 4},
        learned=os.path.join(ROOT, "premixfem_b200", "weights", "fracture16_k6.pmfnet"),
        desc="fracture256: 256^3 unit cells, 200 fractures k=1e4, 5% barriers k=1e-4, p=1|0 on x faces; "
             "16^3 subdomains of 16^3 cells (virtual rank grid 4x4x4, -sd 4), en_lv1=6, en_lv2=4, V-cycle, "
             "rtol 1e-8 (seeded synthetic field, seed 4)",
        sample_n=128, sample_opts={"sd": 4, "vranks": (2, 2, 2), "en_lv1": 6, "en_lv2": 4},
        cpu_opts={"sd": 4, "vranks": (4, 4, 4), "en_lv1": 6, "en_lv2": 4},
    ),
    # the same field through the reference's -use_2level branch: one global coarse problem
    # (24 576 unknowns, banded Cholesky) in place of levels 2 and 3
    "fracture256_2level": dict(
        make=lambda seed: fields.fracture256(256, seed=seed),
        opts={"sd": 4, "pmf_vranks": (4, 4, 4), "en_lv1": 6, "en_lv2": 4, "use_2level": True},
        desc="fracture256 with -use_2level: the global Phi^T A Phi (24 576 unknowns) by the tiled banded "
             "Cholesky, random eigensolver starts",
    ),
    # 60 x 220 x 85 layered channel field (pure Neumann, constant null space), k = 4.
    "layered": dict(
        make=lambda seed: fields.layered(seed=2),
        opts={"pmf_sd": (3, 11, 17), "pmf_vranks": (2, 2, 1), "en_lv1": 4, "en_lv2": 4,
              "ksp_constant_null_space": True},
        desc="layered: 60x220x85 cells of 20x10x2, 35 lognormal layers (sigma 1.5) over 50 layers of sinuous "
             "channels (contrast 1e6), +/-1 injector/producer columns, no-flux walls (-ksp_constant_null_space); "
             "6x22x17 subdomains of 10x10x5 on a 2x2x1 virtual rank grid, en_lv1=4, en_lv2=4; the mixed form "
             "computes the local basis in FP64 (-pmf_eig_precision fp64: with the FP32 eigensolver's 1e-6 "
             "residual the near-zero channel modes are too inexact and CG stalls)",
        mixed_opts={"pmf_eig_precision": "fp64"},
        # the pure-Neumann operator's FP64 CG levels off between 1e-11 and 1e-10 (1e-11 was not reached in
        # 20 000 iterations); solutions are compared modulo constants
        ref_rtol="1e-10", null_space=True,
        cpu_opts={"sd": (3, 11, 17), "vranks": (2, 2, 1), "en_lv1": 4, "en_lv2": 4, "constant_null_space": True},
    ),
    # 512 x 512 x 256 anisotropic GRF with fracture planes, k = 8.
    "large512": dict(
        make=lambda seed: fields.large_frac(512, 512, 256, seed=5),
        opts={"sd": 4, "pmf_vranks": (8, 8, 4), "en_lv1": 8, "en_lv2": 4},
        desc="large512: 512x512x256 unit-cube cells, exp(GRF sigma 3, correlation (0.1, 0.1, 0.02)) with 400 "
             "fracture planes of contrast 1e6, p=0 on z=0, unit source; 32x32x16 subdomains of 16^3 (-sd 4 on an "
             "8x8x4 virtual rank grid), en_lv1=8, en_lv2=4",
    ),
    # 64 independent unit-cube GRF problems of per-axis size U{24..80}, 4 right-hand sides each.
    "batch64": dict(
        batch=True,
        make=lambda seed: fields.grf_batch(count=64, seed=3),
        opts={"en_lv1": 4, "en_lv2": 4},
        desc="batch64: 64 independent unit-cube problems, per-axis cells U{24..80} (seed 3; 8.7 M cells), "
             "k=exp(GRF sigma U[1,3], correlation U[0.05,0.2]), p=0 on x=1; ragged ~8^3 tiles, one virtual rank "
             "per problem, en_lv1=4, en_lv2=4; four right-hand sides each (unit source + 3 N(0,1) fields): one "
             "batched set-up (every phase one launch over all 64 problems' subdomains) and four batched PCG "
             "solves (one CG per problem, all problems per launch)",
        cpu_ref={"value": 181.6, "cores": 8, "setup_s": 113.5, "solve_s": 68.1,
                 "sample": "the C++/OpenMP restatement, FP64, one set-up and four solves per problem, all 64 "
                           "problems, on the 8 cores of the build container (not timed in this run: about 3 min "
                           "of CPU work)"},
    ),
    # 32^3 unit-cube GRF, the small CPU-runnable case.
    "unit_cube_grf32": dict(
        make=lambda seed: fields.unit_cube_grf(32, seed=seed),
        opts={"sd": 4, "en_lv1": 4, "en_lv2": 4},
        desc="unit_cube_grf32: 32^3, k=exp(GRF sigma 2, l 0.1), p=0 on x=1, f=1; 4^3 subdomains of 8^3, k=4",
        sample_n=32, sample_opts={"sd": 4, "en_lv1": 4, "en_lv2": 4},
        cpu_opts={"sd": 4, "en_lv1": 4, "en_lv2": 4},
    ),
}

# ncu DRAM traffic of the level-1 kernel with an iterate (k_ic_apply<float,1,1>), bytes per cell:
# 67 167 488 B read / 2 097 152 cells at 128^3 (profiles/ic_apply_fracture128_mixed.md) plus the
# 8 B/cell FP64 result, which stays in L2 at that size; scaled by the cell count.
IC_APPLY_Y_TRAFFIC_PER_CELL = 67167488 / 2097152 + 8


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "samples": len(sm), "reasons": sorted(reasons)}


def _dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def class_bytes(n, nsub, nrank, nr, n3, k, w):
    """Algorithmic bytes per PCG iteration of each kernel class of pmf_profile_iteration
    (V-cycle, si_lv1 = si_lv2 = 1: one first level-1 visit, one final level-1 visit with
    the iterate, one residual + restriction, one prolongation, two level-2 and one level-3
    coarse solve).  n cells, w bytes per preconditioner value, k basis vectors per subdomain."""
    return {
        # read r (FP64), tx, ty, tz, 1/d; write y
        "lv1_first": n * (8 + 5 * w),
        # read r (FP64), y, tx, ty, tz, diag, 1/d; write the FP64 result
        "lv1_with_y": n * (16 + 6 * w),
        # read r (FP64), y, tx, ty, tz, diag, Phi (k values)
        "resid_restrict": n * (8 + 5 * w + k * w),
        # dense per-rank level-2 inverses (two visits), the level-3 inverse, the coarse blocks
        "coarse": 2 * nrank * nr * nr * 8 + n3 * n3 * 8 + nsub * 7 * k * k * 8,
        # read Phi, y; write y
        "prolong": n * (k + 2) * w,
        # read z, p, tx, ty, tz, diag; write p, w
        "cg_p_update_Ap": n * 64,
        # read x, r, p, w; write x, r
        "cg_x_r_update": n * 48,
        "beta": nsub * 8,
    }


def run_b200(args):
    import torch

    from premixfem_b200 import _native
    from premixfem_b200.solver import DarcySolver

    rank, world, local = _dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    lib = _native.load()
    hbm, bf16, peak_kind = _peaks()

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def maxr(v):
        if not dist:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def measure(name, steps, warmup, headline):
        wl = WORKLOADS[name]
        prob = wl["make"](args.seed + rank)
        M, N, P = prob["mesh"]
        n = M * N * P
        kap = [torch.from_numpy(np.ascontiguousarray(k).ravel()).cuda() for k in prob["kappa"][:1]]
        kx = kap[0]
        src_h = np.ascontiguousarray(prob["source"]).ravel()
        src_d = torch.from_numpy(src_h).cuda()

        def make_solver(form, extra=None):
            o = dict(wl["opts"], pmf_precision="fp64" if form.startswith("fp64") else "mixed")
            if form.startswith("mixed"):
                o.update(wl.get("mixed_opts", {}))
            if form == "mixed" and wl.get("learned"):
                o["pmf_learned"] = wl["learned"]
            if form == "mixed" and headline:
                o["pmf_eig_profile"] = 1  # per-phase CUDA events of the batched eigensolver
            o.update(extra or {})
            s = DarcySolver(prob["dom"], prob["mesh"], options_string(o))
            for f, v in prob["dirichlet"].items():
                s.set_dirichlet(f, v)
            return s

        def device_step(s):
            s.set_kappa(kx, kx, kx)
            s.setup()
            b = torch.empty_like(src_d)
            s.rhs(src_d, b)
            x = torch.empty_like(src_d)
            _, its, rn, reason = s.solve(b, x)
            su, so = s.timing()
            return su, so, its, rn, reason, b, x

        def true_residual(s, b, x):
            ax = torch.empty_like(x)
            s.apply_A(x, ax)
            return float(torch.linalg.norm(b - ax) / torch.linalg.norm(b))

        forms = ["mixed"] + (["mixed_nonet"] if wl.get("learned") else []) + ["fp64"]
        res = {}
        sol = {}
        boxes = None
        for form in forms:
            s = make_solver(form)
            for _ in range(warmup):
                device_step(s)
            barrier()
            steps_l = []
            stages0 = s.stages()
            launches0 = lib.pmf_launch_count()
            with ClockSampler(local) as clk:
                for _ in range(steps):
                    barrier()
                    su, so, its, rn, reason, b, x = device_step(s)
                    barrier()
                    steps_l.append((su, so, its, rn, reason))
            launches = lib.pmf_launch_count() - launches0
            stages1 = s.stages()
            ev1, ks, it1, st1 = s.eigen_lv1()
            lst = (C.c_longlong * 4)()
            net_ms = C.c_double()
            _native.check(lib.pmf_get_learned_stats(s.h, lst, C.byref(net_ms)))
            r = dict(steps=steps_l, launches=launches, clocks=clk.summary(),
                     setup_s=statistics.mean(v[0] for v in steps_l) / 1e3,
                     solve_s=statistics.mean(v[1] for v in steps_l) / 1e3,
                     its=steps_l[-1][2], reason=steps_l[-1][4], rel_residual=true_residual(s, b, x),
                     eig=dict(iters_mean=float(it1.mean()), iters_max=int(it1.max()),
                              status={"converged": int((st1 == 0).sum()), "rounding_floor": int((st1 == 2).sum()),
                                      "max_it": int((st1 == 1).sum())}),
                     ev1=ev1, learned=dict(used=int(lst[0]), fallbacks=int(lst[1]),
                                           net_ms=round(net_ms.value, 3)),
                     # set-up stages per step (ms): local eigensolves, level-2 Galerkin + inverses,
                     # level-3 eigensolve, level-3 Galerkin; the stage timers accumulate over set-ups
                     stages_ms={k: round((stages1[k] - stages0[k]) * 1e3 / max(1, steps), 2)
                                for k in ("su_lv1", "su_lv2_1", "su_lv2_2", "su_lv3_1", "su_lv3_2", "su")})
            if boxes is None:
                boxes = s.subdomains()[0]
            r["t"] = r["setup_s"] + r["solve_s"]
            sol[form] = x
            if form == "mixed" and headline:
                phases = (C.c_double * 8)()
                colcells = C.c_ulonglong()
                _native.check(lib.pmf_get_eig_phases(s.h, phases, C.byref(colcells)))
                r["eig_phases"] = list(phases)
                # per-class kernel times of one PCG iteration on this solve's data
                r["profile"] = s.profile_iteration(reps=5)
                r["info"] = s.info()
                # e2e through the C ABI with host buffers (copies inside the timed region)
                kx_host = torch.from_numpy(np.ascontiguousarray(prob["kappa"][0]).ravel()).pin_memory()
                src_host = torch.from_numpy(src_h).pin_memory()
                x_host = torch.empty(n, dtype=torch.float64).pin_memory()
                b_host = torch.empty(n, dtype=torch.float64).pin_memory()  # the right-hand side comes back here
                e2e = []
                for _ in range(max(1, steps)):
                    barrier()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    s.set_kappa(kx_host.numpy(), kx_host.numpy(), kx_host.numpy())
                    s.setup()
                    s.rhs(src_host.numpy(), b_host.numpy())
                    s.solve(b_host.numpy(), x_host.numpy())
                    e1.record()
                    torch.cuda.synchronize()
                    e2e.append(e0.elapsed_time(e1) / 1e3)
                r["e2e"] = e2e
            res[form] = r
            s.close()
            del s
            gc.collect()
        # FP64 reference solution: the device FP64 form solved to a tight relative residual
        ref_rtol = wl.get("ref_rtol", "1e-13")
        s = make_solver("fp64_ref", {"ksp_rtol": ref_rtol, "ksp_max_it": 20000})
        _, _, its_ref, _, reason_ref, b, xref = device_step(s)
        s.close()
        del s
        if wl.get("null_space"):  # compare modulo constants
            xref = xref - xref.mean()
            sol = {f: v - v.mean() for f, v in sol.items()}
        nref = float(torch.linalg.norm(xref))
        err = {f: float(torch.linalg.norm(sol[f] - xref)) / nref for f in forms}
        out = dict(wl=wl, prob=prob, n=n, res=res, forms=forms, boxes=boxes, err=err,
                   ref=dict(its=its_ref, reason=reason_ref, rtol=ref_rtol, null_space=bool(wl.get("null_space"))))
        del sol, xref, kx, src_d, kap
        gc.collect()
        torch.cuda.empty_cache()
        return out

    def form_summary(r):
        return {"setup_s": round(r["setup_s"], 6), "solve_s": round(r["solve_s"], 6), "total_s": round(r["t"], 6),
                "pcg_iters": r["its"], "reason": r["reason"], "rel_residual": r["rel_residual"],
                "eigensolver": dict(r["eig"], learned_start=r["learned"]), "setup_stages_ms": r["stages_ms"],
                "clocks": r["clocks"]}

    def accuracy(m):
        return {"error_vs_fp64_ref": {f: m["err"][f] for f in m["forms"]},
                "fp64_ref": f"device FP64 form, PCG to relative residual {m['ref']['rtol']} ({m['ref']['its']} "
                            f"iterations, {m['ref']['reason']}); not a direct solve at this size"
                            + ("; solutions compared modulo constants (pure Neumann)" if m["ref"]["null_space"] else "")}

    main_name = args.workload
    m = measure(main_name, args.steps, args.warmup, headline=True)
    wl, n, res = m["wl"], m["n"], m["res"]
    mix, plain = res["mixed"], res["fp64"]
    t_mixed = maxr(mix["t"])
    t_plain = maxr(plain["t"])
    t_e2e = maxr(statistics.mean(mix["e2e"]))

    # roofline: the dominant kernel class of a PCG iteration, timed live
    info = mix["info"]
    k = wl["opts"]["en_lv1"]
    cb = class_bytes(n, info["nsub"], info["nrank"], info["nr"], info["n3"], k, 4)
    prof = mix["profile"]
    per_class = {}
    for c, (ms, nl) in prof.items():
        if nl == 0:
            continue
        per_class[c] = {"ms_per_iteration": round(ms, 4), "launch_groups": nl,
                        "algorithmic_bytes": int(cb[c]),
                        "achieved_gbs": round(cb[c] / (ms * 1e-3) / 1e9, 1) if ms > 0 else None}
        per_class[c]["frac"] = round(per_class[c]["achieved_gbs"] / hbm, 4) if ms > 0 else None
    dom = max((c for c in per_class if c.startswith("lv1") or c in ("resid_restrict", "prolong", "cg_p_update_Ap",
                                                                     "cg_x_r_update")),
              key=lambda c: per_class[c]["ms_per_iteration"])
    d = per_class[dom]
    dom_ms_launch = d["ms_per_iteration"] / d["launch_groups"]
    dom_bytes_launch = cb[dom] / d["launch_groups"]
    tune = _tune_choices(lib) or {}
    lv1_names = {"lv1_with_y": _lv1_kernel(tune, "f32", 1), "lv1_first": _lv1_kernel(tune, "f32", 0)}
    traffic = None
    # the ncu capture is of the natural-order kernel's final visit: its traffic is claimed only for that kernel
    if dom == "lv1_with_y" and IC_APPLY_Y_TRAFFIC_PER_CELL and lv1_names[dom].startswith("k_ic_apply<"):
        traffic = int(IC_APPLY_Y_TRAFFIC_PER_CELL * n)
    iter_ms = sum(v[0] for v in prof.values())
    iter_bytes = sum(cb[c] for c in prof if prof[c][1] > 0)
    biter = n * (104 + 4 * (25 + 6 * k))
    its_m = mix["its"]
    line = {
        "metric": METRIC,
        "value": round(t_mixed, 6),
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_mixed * 1e3, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 PCG / f32 preconditioner (plain form: f64)",
        "data": "synthetic (seeded field generators; the reference's fracture256 / SPE10 data are not distributed)",
        "config": {
            "workload": wl["desc"],
            "cells": n,
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "l2": "inputs larger than L2 (kappa 3 x 134 MB, vectors 134 MB each)",
        },
        "pcg_iters": {"mixed": its_m, "plain_fp64": plain["its"]},
        "setup_s": {"mixed": round(mix["setup_s"], 6), "plain_fp64": round(plain["setup_s"], 6)},
        "solve_s": {"mixed": round(mix["solve_s"], 6), "plain_fp64": round(plain["solve_s"], 6)},
        "plain_fp64_value": round(t_plain, 6),
        "speedup_vs_plain_fp64": round(t_plain / t_mixed, 3),
        "forms": {f: form_summary(res[f]) for f in m["forms"]},
        "accuracy": accuracy(m),
        # host buffers: kappa x3 + source + rhs in (5n doubles); rhs + solution out (2n doubles)
        "e2e": {"value": round(t_e2e, 6), "unit": "s", "h2d_bytes_per_step": int(5 * n * 8),
                "d2h_bytes_per_step": int(2 * n * 8)},
        "gpu_launches": int(mix["launches"] / max(1, args.steps)),
        "roofline": {
            "kernel": {"lv1_with_y": lv1_names["lv1_with_y"] + " (level-1 IC(0) solve with the iterate, final visit)",
                       "lv1_first": lv1_names["lv1_first"] + " (level-1 IC(0) solve, first visit)"}.get(dom, dom),
            "bound": "hbm",
            "achieved": round(dom_bytes_launch / (dom_ms_launch * 1e-3) / 1e9, 1),
            "peak": hbm,
            "unit": "GB/s",
            "frac": round(dom_bytes_launch / (dom_ms_launch * 1e-3) / 1e9 / hbm, 4),
            "traffic": traffic,
            "algorithmic_bytes_per_launch": int(dom_bytes_launch),
            "ms_per_launch": round(dom_ms_launch, 4),
            "peak_kind": peak_kind,
            "timing": "CUDA events on the solver stream around each launch group of one PCG iteration, "
                      "5 repetitions outside the CUDA graph (pmf_profile_iteration)",
        },
        "solve_phase": {
            "model": {"bytes_per_iteration": biter, "formula": "N*[104 + w*(25+6k)], w=4",
                      "achieved_gbs": round(biter * its_m / mix["solve_s"] / 1e9, 1),
                      "frac": round(biter * its_m / mix["solve_s"] / 1e9 / hbm, 4)},
            "launched_kernels": {"bytes_per_iteration": int(iter_bytes), "iteration_ms": round(iter_ms, 4),
                                 "achieved_gbs": round(iter_bytes / (iter_ms * 1e-3) / 1e9, 1),
                                 "frac": round(iter_bytes / (iter_ms * 1e-3) / 1e9 / hbm, 4),
                                 "by_class": per_class},
        },
        "clocks": mix["clocks"],
        "autotune": _tune_choices(lib),
    }
    if "eig_phases" in mix:
        ph = mix["eig_phases"]
        line["lobpcg_phases_ms"] = {"resid_control": round(ph[0], 2), "precond": round(ph[1], 2),
                                    "gram": round(ph[2], 2), "rayleigh_ritz": round(ph[3], 2),
                                    "update": round(ph[4], 2), "a_images": round(ph[5], 2),
                                    "lockstep_iterations": int(ph[6])}
    def measure_batch(name, steps, warmup):
        """A batch workload: per step one batched set-up and four batched solves, per form."""
        from premixfem_b200.solver import BatchSolver
        wl = WORKLOADS[name]
        batch = wl["make"](args.seed)
        problems = [p for p, _ in batch]
        sds = [fields.tiles(p["mesh"]) for p in problems]
        out = {"config": wl["desc"], "cells": int(sum(np.prod(p["mesh"]) for p in problems)),
               "problems": len(problems), "rhs_per_problem": 4, "steps": steps, "warmup": warmup, "forms": {}}
        for form in ("mixed", "fp64"):
            s = BatchSolver(problems, sds, options_string(dict(wl["opts"], pmf_precision=form)))
            kap = [torch.from_numpy(s.pack([p["kappa"][d] for p in problems])).cuda() for d in range(3)]
            srcs = [torch.from_numpy(s.pack([src[j] for _, src in batch])).cuda() for j in range(4)]

            def step():
                s.set_kappa(*kap)
                s.setup()
                su = s.timing()[0]
                so, its_all, reasons = 0.0, [], []
                for j in range(4):
                    b = torch.empty_like(srcs[j])
                    s.rhs(srcs[j], b)
                    x = torch.empty_like(b)
                    _, its, _, rs = s.solve(b, x)
                    so += s.timing()[1]
                    its_all += [int(v) for v in its]
                    reasons += rs
                return su, so, its_all, reasons

            for _ in range(warmup):
                step()
            barrier()
            res = []
            with ClockSampler(local) as clk:
                for _ in range(steps):
                    barrier()
                    res.append(step())
                    barrier()
            su = statistics.mean(r[0] for r in res) / 1e3
            so = statistics.mean(r[1] for r in res) / 1e3
            its_all, reasons = res[-1][2], res[-1][3]
            out["forms"][form] = {"setup_s": round(su, 6), "solve_s": round(so, 6), "total_s": round(su + so, 6),
                                  "pcg_iters_mean": round(float(np.mean(its_all)), 2),
                                  "pcg_iters_max": int(np.max(its_all)),
                                  "converged": int(sum(r == "converged" for r in reasons)), "solves": len(reasons),
                                  "clocks": clk.summary()}
            s.close()
            del kap, srcs, s
            gc.collect()
            torch.cuda.empty_cache()
        out["value"] = round(maxr(out["forms"]["mixed"]["total_s"]), 6)
        out["plain_fp64_value"] = round(maxr(out["forms"]["fp64"]["total_s"]), 6)
        out["speedup_vs_plain_fp64"] = round(out["plain_fp64_value"] / out["value"], 3)
        out["cpu_reference"] = dict(wl["cpu_ref"], unit="s", kind="port")
        out["speedup_vs_cpu_reference"] = round(wl["cpu_ref"]["value"] / out["value"], 1)
        return out

    extras = {}
    # secondary workloads and the CPU baseline belong to the 1-GPU line; a multi-rank (scaling) run
    # measures the headline workload only
    for name in [e for e in args.extra.split(",") if e and e != main_name and world == 1]:
        if WORKLOADS[name].get("batch"):
            try:
                extras[name] = measure_batch(name, 3, 3)
            except Exception as ex:  # a secondary workload never voids the headline line
                extras[name] = {"error": f"{type(ex).__name__}: {ex}"}
            gc.collect()
            continue
        try:
            e = measure(name, 3, 3, headline=False)
            er = e["res"]
            extras[name] = {"config": e["wl"]["desc"], "cells": e["n"], "steps": 3, "warmup": 3,
                            "value": round(maxr(er["mixed"]["t"]), 6),
                            "plain_fp64_value": round(maxr(er["fp64"]["t"]), 6),
                            "speedup_vs_plain_fp64": round(er["fp64"]["t"] / er["mixed"]["t"], 3),
                            "forms": {f: form_summary(er[f]) for f in e["forms"]},
                            "accuracy": accuracy(e)}
            del e
        except Exception as ex:  # a secondary workload never voids the headline line
            extras[name] = {"error": f"{type(ex).__name__}: {ex}"}
        gc.collect()
    if extras:
        line["workloads"] = extras
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, wl, m["prob"], plain["its"])
        line["accuracy"]["local_eigenvalues_sample"] = eig_sample(m)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _lv1_kernel(tune, prec, kind):
    """Name of the level-1 kernel the tuner chose for a visit kind (0: first
    visit, 1: with the iterate, timed in its final-visit form).  Candidates:
    the natural-order kernel at each thread count, then (b2 / b3 in the key)
    the blocked kernel at 512 and 256 threads and its staged form."""
    ty = "float" if prec == "f32" else "double"
    args = f"<{ty},1,1>" if kind else f"<{ty},0,0>"
    for key, (choice, us) in tune.items():
        parts = key.split("|")
        if parts[0] != "ic_apply" or parts[1] != prec or f"y{kind}" not in parts:
            continue
        nblk = int(next((q[1:] for q in parts if q.startswith("b") and q[1:].isdigit()), "0"))
        nnat = len(us) - nblk
        if choice < nnat:
            return "k_ic_apply" + args
        return ("k_ic_apply_blk" if choice - nnat < 2 else "k_ic_apply_stg") + args
    return "k_ic_apply" + args


def _tune_choices(lib):
    """The launch-shape tuner's choices of this process: {kernel|shape: [choice, per-candidate us]}."""
    n = lib.pmf_tune_report(None, 0)
    buf = C.create_string_buffer(n + 1)
    lib.pmf_tune_report(buf, n + 1)
    try:
        table = json.loads(buf.value.decode())
    except ValueError:
        return None
    return {k.rsplit("|", 1)[0]: [v["choice"], v["us"]] for k, v in table.items()}


def eig_sample(m, count=64, seed=12):
    """CPU-baseline leg: local eigenvalues of a seeded sample of subdomains, every GPU form
    against the oracle's exact local GHEP (ARPACK shift-and-invert on each subdomain's crop)."""
    from oracle import pmf_oracle as O

    boxes = m["boxes"]
    k = m["wl"]["opts"]["en_lv1"]
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(len(boxes), size=min(count, len(boxes)), replace=False))
    t0 = time.perf_counter()
    ref = O.local_eigenvalues(m["prob"], boxes[pick], k)
    out = {"subdomains": int(len(pick)), "of": int(len(boxes)), "seed": seed,
           "oracle": "exact local GHEP A_N v = lambda M v per subdomain (ARPACK shift-invert, target -1e-12)",
           "oracle_s": round(time.perf_counter() - t0, 2)}
    for f, r in m["res"].items():
        rel, null = O.eigenvalue_errors(r["ev1"][pick], ref)
        out[f] = {"max_rel_err": rel, "null_mode_abs_err_over_lambda_max": null}
    return out


def _crop(prob, ns):
    """The first ns^3 cells of a workload's field, with its cell size and boundary faces."""
    sl = (slice(0, ns), slice(0, ns), slice(0, ns))
    h = [prob["dom"][i] / prob["mesh"][i] for i in range(3)]
    return dict(prob, mesh=(ns, ns, ns), dom=(h[0] * ns, h[1] * ns, h[2] * ns),
                kappa=tuple(np.ascontiguousarray(k[sl]) for k in prob["kappa"]),
                source=np.ascontiguousarray(prob["source"][sl]))


def cpu_run(wl, prob, crop=False):
    """One FP64 setup + PCG solve of the C++/OpenMP restatement (oracle/cpu_ref) on all host threads.

    crop=False: the full workload (16.7 M cells take about 35 s on 16 cores).
    crop=True: the field cropped to an n_s^3 box with the same subdomain size,
    eigen counts and Dirichlet faces (used for warm-up steps only).
    """
    from oracle.cpu_ref import pmf_cpu as CR

    so = wl["sample_opts"] if crop else wl["cpu_opts"]
    sub = _crop(prob, wl["sample_n"]) if crop else prob
    kw = {k: v for k, v in so.items() if k not in ("sd", "vranks")}
    return CR.solve(sub, sd=so["sd"], vranks=so.get("vranks", (1, 1, 1)), **kw)


def cpu_baseline(args, wl, prob, gpu_its):
    r = cpu_run(wl, prob)
    t = r["setup_s"] + r["solve_s"]
    return {"value": round(t, 3), "unit": "s", "cores": r["threads"], "kind": "port",
            "sample": f"the full workload once: C++/OpenMP FP64 restatement (LOBPCG local eigensolves, FP64 "
                      f"everywhere) on {r['threads']} host threads, setup {r['setup_s']:.2f} s + solve "
                      f"{r['solve_s']:.2f} s, {r['its']} PCG iterations (GPU FP64 form: {gpu_its})",
            "pcg_iters": r["its"], "setup_s": round(r["setup_s"], 3), "solve_s": round(r["solve_s"], 3)}


def run_reference(args):
    rank, world, local = _dist_env()
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]
    if "cpu_opts" not in wl:
        print(json.dumps({"impl": "reference", "unavailable": f"no CPU restatement run is defined for "
                                                              f"{args.workload}"}), flush=True)
        return
    prob = wl["make"](args.seed)
    for _ in range(args.warmup):
        cpu_run(wl, prob, crop="sample_n" in wl)
    vals, r = [], None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = cpu_run(wl, prob)
        vals.append(r["setup_s"] + r["solve_s"])
    wall = time.perf_counter() - t0
    value = statistics.mean(vals)
    cb = {"value": round(value, 3), "unit": "s", "cores": r["threads"], "kind": "port",
          "sample": f"full workload per timed step (warm-up steps on a {wl.get('sample_n', 'full')}^3 crop): C++/OpenMP "
                    f"FP64 restatement on {r['threads']} host threads, {r['its']} PCG iterations, last step setup "
                    f"{r['setup_s']:.2f} s + solve {r['solve_s']:.2f} s",
          "wall_s": round(wall, 2)}
    line = {"metric": METRIC, "value": round(value, 3), "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(value * 1e3, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["desc"]}, "impl": "reference", "cpu_baseline": cb,
            "pcg_iters": r["its"],
            "e2e": {"value": round(value, 3), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fracture256",
                    choices=sorted(k for k, v in WORKLOADS.items() if not v.get("batch")))
    ap.add_argument("--extra", default="fracture256_2level,layered,large512,batch64",
                    help="secondary workloads measured after the headline (comma separated, '' for none)")
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
