"""The reference's own experiment driver against this repository's headers.

src/Expe_scal.c (the cross-field driver) is compiled with its include list
swapped for "PreMixFEM_3D.h" and nothing else changed, with implicit function
declarations as errors, and linked against libpremixfem_b200.so.  Without a
GPU the program must get as far as PC_init and stop there with the library's
"no CUDA device" error (76); with one it runs to completion.  The source is
read where the reference checkout lies (PMF_REFERENCE_SRC, default the
reference's src/ directory next to this repository's parent); the test skips
when it is absent, and nothing from it is kept.

Not covered: src/test.c calls a six-argument PC_init that the reference's own
header no longer declares, and src/Expe_frac.c reads its permeability through
PETSc's HDF5 viewer, which the compatibility layer does not provide.
"""
import os
import re
import shutil
import subprocess

import pytest

from premixfem_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.environ.get("PMF_REFERENCE_SRC", os.path.join(os.path.dirname(ROOT), "reference", "src"))


def _swap_includes(text):
    """PETSc / SLEPc / MPI headers and the reference's own header out, this
    repository's drop-in header in."""
    text = re.sub(r'#include\s*[<"](petsc|slepc|mpi)[^>"]*[>"]', r"/* \g<0> */", text)
    text = re.sub(r'#include\s*"PreMixFEM_3D.h"', "", text)
    return '#include "PreMixFEM_3D.h"\n' + text


def test_expe_scal_builds_and_reaches_the_device(tmp_path):
    src = os.path.join(SRC, "Expe_scal.c")
    if not os.path.exists(src):
        pytest.skip("the reference checkout is not available")
    if shutil.which("gcc") is None:
        pytest.skip("gcc is not available")
    lib = _native.load()  # builds nothing: the in-tree library must exist
    libdir = os.path.join(ROOT, "premixfem_b200", "_lib")
    c = tmp_path / "Expe_scal.c"
    c.write_text(_swap_includes(open(src).read()))
    exe = tmp_path / "expe_scal"
    cmd = ["gcc", "-std=gnu99", "-O1", "-Werror=implicit-function-declaration", "-I", os.path.join(ROOT, "include"),
           str(c), "-L", libdir, "-lpremixfem_b200", f"-Wl,-rpath,{libdir}", "-lm", "-o", str(exe)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    r = subprocess.run([str(exe), "-size", "8", "-cr", "2"], capture_output=True, text=True, timeout=600)
    out = r.stdout + r.stderr
    if lib.pmf_device_count() > 0:
        assert r.returncode == 0, out
    else:
        assert r.returncode != 0 and "no CUDA device available" in out, out
        assert "PC_init" in out, out
