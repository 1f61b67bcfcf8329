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


def test_library_exports_reference_interface_and_petsc_subset():
    """PreMixFEM_3D.h (the reference's entry points) and pmf_petsc_compat.h."""
    lib = _native.load()
    ref = declared_functions("PreMixFEM_3D.h")
    assert set(ref) >= {"PC_init", "PC_setup", "PC_create_A", "PC_apply_vec", "PC_get_range",
                        "PC_print_info", "PC_print_stat", "PC_final", "PC_final_default", "_PC_setup"}
    compat = declared_functions("pmf_petsc_compat.h")
    assert {"KSPSolve", "DMDAVecGetArray", "MatMult", "PCShellSetApply"} <= set(compat)
    for n in ref + compat:
        assert hasattr(lib, n), f"missing export {n}"


def test_every_header_is_covered():
    headers = sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h"))
    assert headers == ["PreMixFEM_3D.h", "pmf_b200.h", "pmf_petsc_compat.h"]


def test_option_errors_come_before_the_device():
    """pmf_create checks its options on the host first: a malformed option is
    argument error 62 with or without a GPU; well-formed options get as far as
    the device (0 with a GPU, 76 without one)."""
    import ctypes as C

    lib = _native.load()
    dom = (C.c_double * 3)(1.0, 1.0, 1.0)
    mesh = (C.c_int * 3)(8, 8, 8)

    def create(opts):
        h = C.c_void_p()
        rc = lib.pmf_create(C.cast(dom, C.c_void_p), C.cast(mesh, C.c_void_p), opts.encode(), C.byref(h))
        if rc == 0:
            lib.pmf_destroy(h)
        return rc

    bad = ["-eg_op 7", "-pmf_precision half", "-ksp_constant_null_space maybe", "-pmf_eig_rel_floor 1.5",
           "-pmf_eig_rel_floor -0.1", "-pmf_learned", "-pmf_eig_guard -1", "-pmf_eig_ctas -4",
           "-pmf_lv1_kernel fast"]
    for opts in bad:
        assert create("-sd 2 " + opts) == 62, opts
    good = ["", "-ksp_constant_null_space", "-ksp_constant_null_space false", "-pmf_eig_rel_floor 1e-4",
            "-pmf_eig_init 1 -pmf_precision mixed", "-use_2level -no_shift_A_cc", "-pmf_lv1_kernel staged",
            "-pmf_eig_guard 0"]
    for opts in good:
        assert create("-sd 2 " + opts) in (0, 76), opts


def test_batch_layout_and_argument_checks():
    """Host side of pmf_batch_create: argument errors come before the device
    (62 with or without a GPU), and the shared-mesh packing round-trips."""
    import ctypes as C

    import numpy as np

    from premixfem_b200 import _native
    from premixfem_b200.solver import BatchSolver

    lib = _native.load()
    dom = np.ones(6)
    mesh = np.array([8, 8, 8, 0, 8, 8], dtype=np.int32)
    sd = np.full(6, 2, dtype=np.int32)
    h = C.c_void_p()
    assert lib.pmf_batch_create(2, dom.ctypes.data_as(C.c_void_p), mesh.ctypes.data_as(C.c_void_p),
                                sd.ctypes.data_as(C.c_void_p), b"", C.byref(h)) == 62
    assert lib.pmf_batch_create(0, None, None, None, b"", C.byref(h)) == 62
    mesh[3] = 8
    assert lib.pmf_batch_create(2, dom.ctypes.data_as(C.c_void_p), mesh.ctypes.data_as(C.c_void_p),
                                sd.ctypes.data_as(C.c_void_p), b"-eg_op 9", C.byref(h)) == 62
    # packing on the shared mesh (no device needed): the layout the library reports
    s = BatchSolver.__new__(BatchSolver)
    s.meshes = [(3, 4, 2), (5, 2, 3)]
    s.mesh = (5, 4, 2 + 1 + 3)
    s.z0 = [0, 3]
    a = [np.arange(24.0), 100 + np.arange(30.0)]
    v = s.pack(a)
    assert v.size == 5 * 4 * 6 and np.count_nonzero(v) == 24 + 30 - 1
    back = s.unpack(v)
    assert all(np.array_equal(x, y) for x, y in zip(a, back))
