"""ctypes front end of the C++/OpenMP CPU restatement (pmf_cpu.cpp).

TEST INFRASTRUCTURE and the timed CPU baseline only: imported by tests/ and by
the CPU legs of bench.py, never by the library.  `build()` compiles
libpmf_cpu.so beside this file with g++ (-O3 -fopenmp); `solve()` takes the
same problem dicts as oracle/pmf_oracle.py and premixfem_b200.fields.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libpmf_cpu.so")
SRC = os.path.join(HERE, "pmf_cpu.cpp")
FACES = ("x-", "x+", "y-", "y+", "z-", "z+")

_lib = None


def build(force=False):
    """Compile libpmf_cpu.so when it is missing or older than its source."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    subprocess.run(["make", "-s"] + (["-B"] if force else []) + ["-C", HERE, "libpmf_cpu.so"], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        lib.pmf_cpu_solve.argtypes = [ip, dp, dp, dp, dp, dp, ip, dp, ip, dp, dp, dp]
        lib.pmf_cpu_solve.restype = C.c_int
        _lib = lib
    return _lib


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def solve(problem, sd=(2, 2, 2), vranks=(1, 1, 1), en_lv1=4, en_lv2=4, si_lv1=1, si_lv2=1, use_W_cycle=False,
          eg_op=0, rtol=1e-8, max_it=10000, eig_tol=1e-8, eig_max_it=300, eig_sigma=1e-2, threads=0,
          constant_null_space=False, eig_rel_floor=0.0, eb_lv1=-1.0, eb_lv2=-1.0, no_shift_A_cc=False,
          use_2level=False, use_full_Cholesky_lv1=False, sources=None):
    """Setup + PCG solve.  Returns dict(x, its, setup_s, solve_s, threads, eig_its_mean,
    eig_its_max, eig_unconverged, rnorm, r0, n3).

    ``sources``: several right-hand sides (arrays shaped like problem["source"])
    solved after one set-up instead of problem["source"]; then x has one row per
    source, solve_s covers them all, its / rnorm / r0 are the first one's, and
    its_sum / its_max cover all."""
    lib = load()
    M, N, P = problem["mesh"]
    if isinstance(sd, int):
        sd = (2, 2, 2) if sd == 1 else (sd, sd, sd)  # a single subdomain is reset to 2 (:1718-1721)
    kx, ky, kz = (np.ascontiguousarray(k, dtype=np.float64).ravel() for k in problem["kappa"])
    srcs = [problem["source"]] if sources is None else list(sources)
    nrhs = len(srcs)
    src = np.ascontiguousarray(np.stack([np.asarray(v, dtype=np.float64).ravel() for v in srcs]))
    dir_on = np.zeros(6, dtype=np.int32)
    dir_val = np.zeros(6, dtype=np.float64)
    for f, v in problem.get("dirichlet", {}).items():
        dir_on[FACES.index(f)] = 1
        dir_val[FACES.index(f)] = v
    mesh = np.array([M, N, P], dtype=np.int32)
    dom = np.array(problem["dom"], dtype=np.float64)
    iopt = np.array(list(sd) + list(vranks) + [en_lv1, en_lv2, si_lv1, si_lv2, int(bool(use_W_cycle)), max_it,
                                               eig_max_it, eg_op, threads, int(bool(constant_null_space)),
                                               int(bool(no_shift_A_cc)), int(bool(use_2level)),
                                               int(bool(use_full_Cholesky_lv1)), nrhs], dtype=np.int32)
    dopt = np.array([rtol, eig_tol, eig_sigma, eig_rel_floor, eb_lv1, eb_lv2], dtype=np.float64)
    x = np.zeros((nrhs, M * N * P))
    info = np.zeros(12)
    rc = lib.pmf_cpu_solve(_iptr(mesh), _dptr(dom), _dptr(kx), _dptr(ky), _dptr(kz), _dptr(src), _iptr(dir_on),
                           _dptr(dir_val), _iptr(iopt), _dptr(dopt), _dptr(x), _dptr(info))
    if rc != 0:
        raise ValueError(f"pmf_cpu_solve rejected the arguments ({rc})")
    return {"x": x[0] if sources is None else x, "its": int(info[0]), "its_sum": int(info[10]),
            "its_max": int(info[11]), "setup_s": float(info[1]), "solve_s": float(info[2]),
            "threads": int(info[3]), "eig_its_mean": float(info[4]), "eig_its_max": int(info[5]),
            "eig_unconverged": int(info[6]), "rnorm": float(info[7]), "r0": float(info[8]), "n3": int(info[9])}
