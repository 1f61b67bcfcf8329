"""The reference-style C driver (tests/c/darcy_driver.c) over PreMixFEM_3D.h.

CPU: the driver compiles with gcc against the headers alone and links
against libpremixfem_b200.so.  GPU: it runs the cross-channel problem through
PC_init / PC_create_A / KSPSolve with the PCSHELL, and its iteration count and
solution match the oracle's PCG (iterations within +-1 under -no_shift_A_cc;
solution within 1e-8 relative L2 of an FP64 direct solve of the same
normalised system, with the constant null-space component removed since the
operator is pure Neumann).
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from oracle import pmf_oracle as O
from premixfem_b200 import _native, fields

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "darcy_driver.c")


def _compile(tmp_path):
    gcc = shutil.which("gcc") or shutil.which("cc")
    if gcc is None:
        pytest.skip("no C compiler")
    _native.load()  # builds nothing; fails loudly if the library is missing
    exe = str(tmp_path / "darcy_driver")
    libdir = os.path.dirname(_native.LIB_PATH)
    cmd = [gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", libdir, "-lpremixfem_b200", f"-Wl,-rpath,{libdir}", "-lm", "-o", exe]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    return exe


def test_driver_compiles_against_headers(tmp_path):
    exe = _compile(tmp_path)
    assert os.path.exists(exe)


def _run(exe, args, tmp_path):
    out = str(tmp_path / "x.bin")
    p = subprocess.run([exe] + args + ["-out", out], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    its = int(re.search(r"iterations=(\d+)", p.stdout).group(1))
    return p.stdout, its, np.fromfile(out, dtype=np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("shift", [False, True], ids=["no_shift_A_cc", "nil_shift"])
def test_driver_matches_oracle(tmp_path, precision, shift):
    """Pure Neumann: with the default +NIL shift of the level-3 matrix the
    constant mode is amplified by 1/NIL = 1e12, so the iteration count at a
    tight tolerance depends on rounding (the oracle itself moves between 26
    and 38 iterations when the source is perturbed by 1e-15 relative).  The
    iteration count is therefore compared under -no_shift_A_cc, where the
    null direction is dropped deterministically; the shifted run must still
    converge to the same solution."""
    exe = _compile(tmp_path)
    size, cr = 16, 3
    args = ["-size", str(size), "-cr", str(cr), "-sd", "2", "-en_lv1", "4", "-en_lv2", "4",
            "-pmf_vranks", "1,2,2", "-ksp_rtol", "1e-10", "-pmf_precision", precision]
    if not shift:
        args.append("-no_shift_A_cc")
    stdout, its, x = _run(exe, args, tmp_path)
    assert "Linear solve converged due to CONVERGED_RTOL" in stdout
    assert "eigen_num_lv1_range=[" in stdout and "size_mat_lv3=" in stdout

    prob = fields.cross(size, cr)
    prob["source"] = prob["source"] / np.linalg.norm(prob["source"])
    o = O.Options()
    o.sd, o.vranks, o.en_lv1, o.en_lv2, o.rtol = (2, 2, 2), (1, 2, 2), 4, 4, 1e-10
    o.no_shift_A_cc = not shift
    ref = O.solve(prob, o)
    if not shift:
        assert abs(its - ref["its"]) <= 1, (its, ref["its"])
    xd = O.direct_solve(ref["op"], ref["b"])
    xd = xd - xd.mean()
    xc = x - x.mean()
    assert np.linalg.norm(xc - xd) <= 1e-8 * np.linalg.norm(xd)


@pytest.mark.gpu
def test_driver_plain_cg_host_path(tmp_path):
    """-petsc_default: PETSc's CG recurrence on the host over the device MatMult."""
    exe = _compile(tmp_path)
    stdout, its, x = _run(exe, ["-size", "8", "-cr", "1", "-ksp_rtol", "1e-10", "-petsc_default"], tmp_path)
    prob = fields.cross(8, 1)
    prob["source"] = prob["source"] / np.linalg.norm(prob["source"])
    op = O.Operator(prob)
    b = op.rhs()
    assert np.linalg.norm(op.A @ x - b) <= 1e-9 * np.linalg.norm(b)
    ref = O.pcg(op.A, b, lambda v: v.copy(), rtol=1e-10)
    assert abs(its - ref[1]) <= 1
