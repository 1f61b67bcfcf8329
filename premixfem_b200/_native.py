"""ctypes binding of libpremixfem_b200.so (include/pmf_b200.h).

There is no fallback: if the library is missing or cannot be loaded, every
entry point raises.  Build it with ``python -m premixfem_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libpremixfem_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p

# name -> (restype, argtypes); pointer arguments are passed as c_void_p so
# host numpy buffers and device addresses go through the same signature.
SIGNATURES = {
    "pmf_create": (C.c_int, [_vp, _vp, C.c_char_p, C.POINTER(C.c_void_p)]),
    "pmf_destroy": (C.c_int, [_vp]),
    "pmf_set_kappa": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int]),
    "pmf_set_dirichlet": (C.c_int, [_vp, C.c_int, C.c_double]),
    "pmf_setup": (C.c_int, [_vp]),
    "pmf_rhs": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "pmf_apply_A": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "pmf_pc_apply": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "pmf_solve": (C.c_int, [_vp, _vp, _vp, C.c_int, _ip, _dp, _ip]),
    "pmf_get_info": (C.c_int, [_vp, _vp]),
    "pmf_get_eigen_lv1": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "pmf_get_eigen_lv2": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pmf_get_subdomains": (C.c_int, [_vp, _vp, _vp]),
    "pmf_get_phi": (C.c_int, [_vp, _vp]),
    "pmf_get_coarse_blocks": (C.c_int, [_vp, _vp]),
    "pmf_get_stages": (C.c_int, [_vp, _vp]),
    "pmf_get_timing": (C.c_int, [_vp, _dp, _dp]),
    "pmf_net_create": (C.c_int, [C.c_ulonglong, C.POINTER(C.c_void_p)]),
    "pmf_net_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "pmf_net_save": (C.c_int, [_vp, C.c_char_p]),
    "pmf_net_destroy": (C.c_int, [_vp]),
    "pmf_net_params": (C.c_int, [_vp]),
    "pmf_net_layer_info": (C.c_int, [C.c_int, _vp]),
    "pmf_net_forward": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "pmf_net_backward": (C.c_int, [_vp, _vp, C.c_int]),
    "pmf_net_adam": (C.c_int, [_vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]),
    "pmf_net_get_weights": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "pmf_net_set_weights": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "pmf_net_get_grads": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "pmf_net_loss": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp]),
    "pmf_learned_patches": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pmf_get_learned_stats": (C.c_int, [_vp, _vp, _dp]),
    "pmf_get_eig_phases": (C.c_int, [_vp, _vp, C.POINTER(C.c_ulonglong)]),
    "pmf_profile_iteration": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "pmf_batch_create": (C.c_int, [C.c_int, _vp, _vp, _vp, C.c_char_p, C.POINTER(C.c_void_p)]),
    "pmf_batch_info": (C.c_int, [_vp, _vp, _vp]),
    "pmf_batch_set_dirichlet": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double]),
    "pmf_batch_solve": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp, _vp, _vp]),
    "pmf_residual_noalloc": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "pmf_tune_report": (C.c_int, [C.c_char_p, C.c_int]),
    "pmf_launch_count": (C.c_ulonglong, []),
    "pmf_last_error": (C.c_char_p, []),
    "pmf_device_count": (C.c_int, []),
}

_lib = None


def load():
    """Load the library once; raises OSError with build instructions if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} not found: build it with `python -m premixfem_b200.build` "
                      "(the CUDA library is required; there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class PmfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"premixfem_b200 error {code}: {msg}")
        self.code = code


def check(code):
    if code != 0:
        raise PmfError(code, load().pmf_last_error().decode(errors="replace"))
