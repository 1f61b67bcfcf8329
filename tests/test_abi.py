"""The C ABI library loads and exports every symbol its headers declare (no GPU)."""
import os
import re

from premixfem_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src, flags=re.M)
    return [n for n in names if not n.startswith(("if", "while", "for", "return"))]


def test_library_loads_and_exports_flat_abi():
    lib = _native.load()
    names = declared_functions("pmf_b200.h")
    assert "pmf_solve" in names and "pmf_create" in names
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    assert set(names) == set(_native.SIGNATURES), "ctypes signature table out of sync with pmf_b200.h"


def test_no_device_calls_fail_cleanly_without_gpu():
    lib = _native.load()
    # pmf_device_count never faults; on a CPU-only host it reports 0
    assert lib.pmf_device_count() >= 0
