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

  value   mixed/learned form, inputs resident in HBM (kappa and rhs on the device)
  e2e     mixed form through the C ABI with host buffers (host->device copy
          of kappa and source, device->host copy of the solution, inside the
          timed region)
  plain   plain FP64 form, same workload, for the speed-up the metric names

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
             "16^3 subdomains of 16^3 cells (virtual rank grid 4x4x4, -sd 4), en_lv1=6, en_lv2=4, V-cycle; "
             "mixed form with the learned eigensolver start (network trained on seeds 101-110, this field is "
             "seed 4)",
        sample_n=128, sample_opts={"sd": 4, "vranks": (2, 2, 2), "en_lv1": 6, "en_lv2": 4},
        cpu_opts={"sd": 4, "vranks": (4, 4, 4), "en_lv1": 6, "en_lv2": 4},
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

# Algorithmic bytes per cell of the FP64 operator kernel k_spmv (y = A x):
# reads x, tx, ty, tz, diag (5 x 8 B), writes y (8 B).
SPMV_BYTES_PER_CELL = 6 * 8


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
    wl = WORKLOADS[args.workload]
    prob = wl["make"](args.seed + rank)
    M, N, P = prob["mesh"]
    n = M * N * P
    kx = torch.from_numpy(np.ascontiguousarray(prob["kappa"][0]).ravel()).cuda()
    src_h = np.ascontiguousarray(prob["source"]).ravel()
    src_d = torch.from_numpy(src_h).cuda()
    kx_host = torch.from_numpy(np.ascontiguousarray(prob["kappa"][0]).ravel()).pin_memory()
    src_host = torch.from_numpy(src_h).pin_memory()
    x_host = torch.empty(n, dtype=torch.float64).pin_memory()

    def make_solver(prec):
        o = dict(wl["opts"], pmf_precision=prec)
        if prec == "mixed" and wl.get("learned"):
            o["pmf_learned"] = wl["learned"]
        if prec == "mixed":
            o["pmf_eig_profile"] = 1  # per-phase CUDA events of the batched eigensolver (roofline below)
        s = DarcySolver(prob["dom"], prob["mesh"], options_string(o))
        for f, v in prob["dirichlet"].items():
            s.set_dirichlet(f, v)
        return s

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

    def device_step(s):
        s.set_kappa(kx, kx, kx)
        s.setup()
        b = torch.empty_like(src_d)
        s.rhs(src_d, b)
        x = torch.empty_like(src_d)
        _, its, rn, reason = s.solve(b, x)
        su, so = s.timing()
        return su, so, its, rn, reason, b, x

    results = {}
    for prec in ("mixed", "fp64"):
        s = make_solver(prec)
        for _ in range(args.warmup):
            device_step(s)
        barrier()
        steps = []
        launches0 = lib.pmf_launch_count()
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                barrier()
                su, so, its, rn, reason, b, x = device_step(s)
                barrier()
                steps.append((su, so, its, rn, reason))
        launches = lib.pmf_launch_count() - launches0
        stages = s.stages()
        ev1, ks, it1, st1 = s.eigen_lv1()
        lst = (C.c_longlong * 4)()
        net_ms = C.c_double()
        _native.check(lib.pmf_get_learned_stats(s.h, lst, C.byref(net_ms)))
        phases = (C.c_double * 8)()
        colcells = C.c_ulonglong()
        _native.check(lib.pmf_get_eig_phases(s.h, phases, C.byref(colcells)))
        bn = float(torch.linalg.norm(b))
        res = float(torch.linalg.norm(b - torch.from_numpy(s.apply_A(x.cpu().numpy())).cuda())) / bn
        results[prec] = dict(steps=steps, launches=launches, clocks=clk.summary(), stages=stages,
                             eig_iters_mean=float(it1.mean()), eig_iters_max=int(it1.max()),
                             eig_iters_sum=int(it1.sum()), cells_per_sub=n / len(it1),
                             eig_unconverged=int((st1 != 0).sum()), rel_residual=res, x=x.cpu().numpy(),
                             learned=dict(used=int(lst[0]), fallbacks=int(lst[1]), net_ms=round(net_ms.value, 3)),
                             eig_phases=list(phases), eig_colcells=int(colcells.value))
        if prec == "mixed":
            # e2e through the C ABI with host buffers (copies inside the timed region)
            e2e = []
            for _ in range(max(1, args.steps)):
                barrier()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                s.set_kappa(kx_host.numpy(), kx_host.numpy(), kx_host.numpy())
                s.setup()
                bh = s.rhs(src_host.numpy())
                s.solve(bh, x_host.numpy())
                e1.record()
                torch.cuda.synchronize()
                e2e.append(e0.elapsed_time(e1) / 1e3)
            results["e2e"] = e2e
            # live per-kernel timing of the PCG operator kernel for the solve-phase roofline
            results["spmv_ms"] = time_spmv(s, n)
        s.close()

    mixed = results["mixed"]["steps"]
    plain = results["fp64"]["steps"]
    t_mixed = maxr(statistics.mean(su + so for su, so, *_ in mixed) / 1e3)
    t_plain = maxr(statistics.mean(su + so for su, so, *_ in plain) / 1e3)
    t_e2e = maxr(statistics.mean(results["e2e"]))
    su_m = statistics.mean(x[0] for x in mixed) / 1e3
    so_m = statistics.mean(x[1] for x in mixed) / 1e3
    su_p = statistics.mean(x[0] for x in plain) / 1e3
    so_p = statistics.mean(x[1] for x in plain) / 1e3
    its_m = mixed[-1][2]
    its_p = plain[-1][2]
    xdiff = float(np.linalg.norm(results["mixed"]["x"] - results["fp64"]["x"]) / np.linalg.norm(results["fp64"]["x"]))
    hbm, bf16, peak_kind = _peaks()
    # dominant kernel of the step: the batched local eigensolver (stage su_lv2_1)
    st = results["mixed"]["stages"]
    eig_s = st["su_lv2_1"] / (args.steps + args.warmup)
    spmv_ms = results["spmv_ms"]
    # dominant kernel of the step: the batched eigensolver's basis update k_eb_update<float>
    # (X <- [X W P] Y, P <- [W P] Y per subdomain).  Algorithmic bytes per subdomain-iteration:
    # read the nS basis columns and write X and P (2m columns), 4 bytes per FP32 value; the library
    # counts sum(nS x cells) over subdomain-iterations (colcells) and times the phase with events.
    m_blk = wl["opts"]["en_lv1"] + 2
    lob_sub_iters = results["mixed"]["eig_iters_sum"]
    ph = results["mixed"]["eig_phases"]
    upd_bytes = 4.0 * (results["mixed"]["eig_colcells"] + 2 * m_blk * results["mixed"]["cells_per_sub"] * lob_sub_iters)
    upd_s = ph[4] * 1e-3
    biter = n * (104 + 4 * (25 + 6 * wl["opts"]["en_lv1"]))
    spmv_gbs = SPMV_BYTES_PER_CELL * n / (spmv_ms * 1e-3) / 1e9
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
        "pcg_iters": {"mixed": its_m, "plain_fp64": its_p},
        "setup_s": {"mixed": round(su_m, 6), "plain_fp64": round(su_p, 6)},
        "solve_s": {"mixed": round(so_m, 6), "plain_fp64": round(so_p, 6)},
        "plain_fp64_value": round(t_plain, 6),
        "speedup_vs_plain_fp64": round(t_plain / t_mixed, 3),
        "rel_residual": {"mixed": results["mixed"]["rel_residual"], "plain_fp64": results["fp64"]["rel_residual"]},
        "solution_rel_diff_mixed_vs_fp64": xdiff,
        "eigensolver": {"iters_mean": results["mixed"]["eig_iters_mean"], "iters_max": results["mixed"]["eig_iters_max"],
                        "unconverged": results["mixed"]["eig_unconverged"],
                        "plain_fp64_iters_mean": results["fp64"]["eig_iters_mean"],
                        "plain_fp64_iters_max": results["fp64"]["eig_iters_max"],
                        "learned_start": results["mixed"]["learned"]},
        # host buffers: kappa x3 + source + rhs in (5n doubles); rhs + solution out (2n doubles)
        "e2e": {"value": round(t_e2e, 6), "unit": "s", "h2d_bytes_per_step": int(5 * n * 8),
                "d2h_bytes_per_step": int(2 * n * 8)},
        "gpu_launches": int(results["mixed"]["launches"] / max(1, args.steps)),
        "roofline": {
            "kernel": "k_eb_update<float> (batched LOBPCG basis update, largest single kernel of the step)",
            "bound": "hbm",
            "achieved": round(upd_bytes / upd_s / 1e9, 1) if upd_s > 0 else None,
            "peak": hbm,
            "unit": "GB/s",
            "frac": round(upd_bytes / upd_s / 1e9 / hbm, 4) if upd_s > 0 else None,
            "traffic": None,
            "bytes_per_step": upd_bytes,
            "time_s_per_step": round(upd_s, 6),
            "peak_kind": peak_kind,
        },
        "lobpcg_phases_ms": {"resid_control": round(ph[0], 2), "precond": round(ph[1], 2), "gram": round(ph[2], 2),
                             "rayleigh_ritz": round(ph[3], 2), "update": round(ph[4], 2),
                             "a_images": round(ph[5], 2), "lockstep_iterations": int(ph[6]),
                             "eigen_stage_s": round(eig_s, 6)},
        "roofline_solve_model": {
            "phase": "PCG solve (all kernels), algorithmic bytes B_iter = N*[104 + w*(25+6k)], w=4, k=6",
            "bound": "hbm",
            "achieved": round(biter * its_m / so_m / 1e9, 1),
            "peak": hbm,
            "unit": "GB/s",
            "frac": round(biter * its_m / so_m / 1e9 / hbm, 4),
            "bytes_per_iteration": biter,
        },
        "roofline_solve": {
            "kernel": "k_spmv (7-point FP64 operator, y = A x)",
            "bound": "hbm",
            "achieved": round(spmv_gbs, 1),
            "peak": hbm,
            "unit": "GB/s",
            "frac": round(spmv_gbs / hbm, 4),
            "traffic": None,
            "bytes_per_cell": SPMV_BYTES_PER_CELL,
            "peak_kind": peak_kind,
        },
        "clocks": results["mixed"]["clocks"],
        "autotune": _tune_choices(lib),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, wl, prob, its_p)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


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


def time_spmv(s, n):
    """Average duration of the FP64 PCG operator kernel, timed with CUDA events on the solver stream."""
    import torch
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(3):
        s.apply_A(x, y)
    torch.cuda.synchronize()
    reps = 20
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        s.apply_A(x, y)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


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
    return CR.solve(sub, sd=so["sd"], vranks=so.get("vranks", (1, 1, 1)), en_lv1=so["en_lv1"], en_lv2=so["en_lv2"])


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
    prob = wl["make"](args.seed)
    for _ in range(args.warmup):
        cpu_run(wl, prob, crop=True)
    vals, r = [], None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = cpu_run(wl, prob)
        vals.append(r["setup_s"] + r["solve_s"])
    wall = time.perf_counter() - t0
    value = statistics.mean(vals)
    cb = {"value": round(value, 3), "unit": "s", "cores": r["threads"], "kind": "port",
          "sample": f"full workload per timed step (warm-up steps on a {wl['sample_n']}^3 crop): C++/OpenMP FP64 "
                    f"restatement on {r['threads']} host threads, {r['its']} PCG iterations, last step setup "
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
    ap.add_argument("--workload", default="fracture256", choices=sorted(WORKLOADS))
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
