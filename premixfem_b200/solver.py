"""Python host API over the C ABI, mirroring the reference's PC_* interface.

The reference drives its preconditioner through PETSc (src/Expe_scal.c:66-160):
PC_init -> user builds kappa -> PC_create_A -> KSP with a PCSHELL whose set-up
and apply are PC_setup / PC_apply_vec -> KSPSolve -> PC_print_stat ->
PC_final.  ``PCCtx`` and the ``PC_*`` functions below keep those names and
that order; ``DarcySolver`` is the same thing as one object.

All compute runs in libpremixfem_b200.so on the GPU.  Vectors may be numpy
arrays (host) or objects exposing ``data_ptr()`` (torch CUDA tensors, float64,
contiguous), which are passed to the library as device pointers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native

FACE_IDS = {"x-": 0, "x+": 1, "y-": 2, "y+": 3, "z-": 4, "z+": 5}
STAGE_NAMES = ("su_lv1", "su_lv2_1", "su_lv2_2", "su_lv3_1", "su_lv3_2", "av_lv1", "av_lv2", "av_lv3", "su", "av")
REASONS = {1: "converged", 2: "diverged_its", 3: "diverged_indefinite", 4: "diverged_nanorinf",
           5: "converged_atol"}


def options_string(opts=None, **kw):
    """Build a PETSc-style option string from a dict ({'sd': 4, 'pmf_vranks': (2, 2, 2), 'use_W_cycle': True})."""
    d = dict(opts or {})
    d.update(kw)
    parts = []
    for k, v in d.items():
        if v is None or v is False:
            continue
        if v is True:
            parts.append(f"-{k}")
        elif isinstance(v, (tuple, list)):
            parts.append(f"-{k} {','.join(str(int(x)) for x in v)}")
        else:
            parts.append(f"-{k} {v}")
    return " ".join(parts)


def _ptr(a, dtype=np.float64, writable=False):
    """(pointer, on_device, keepalive) for a numpy array or a CUDA tensor."""
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        return C.c_void_p(a.data_ptr()), 1, a
    arr = np.ascontiguousarray(a, dtype=dtype)
    if writable and arr is not a:
        raise ValueError("output array must be a contiguous float64 numpy array")
    return arr.ctypes.data_as(C.c_void_p), 0, arr


class DarcySolver:
    """One preconditioned CG solver on one GPU (a PCCtx plus its KSP)."""

    def __init__(self, dom, mesh, options=""):
        self.lib = _native.load()
        self.mesh = tuple(int(v) for v in mesh)
        self.dom = tuple(float(v) for v in dom)
        if isinstance(options, dict):
            options = options_string(options)
        self.options = options
        h = C.c_void_p()
        d = (C.c_double * 3)(*self.dom)
        m = (C.c_int * 3)(*self.mesh)
        _native.check(self.lib.pmf_create(C.cast(d, C.c_void_p), C.cast(m, C.c_void_p), options.encode(), C.byref(h)))
        self.h = h
        self.n = self.mesh[0] * self.mesh[1] * self.mesh[2]

    @classmethod
    def from_problem(cls, problem, options=""):
        s = cls(problem["dom"], problem["mesh"], options)
        kx, ky, kz = problem["kappa"]
        s.set_kappa(kx, ky, kz)
        for face, val in problem.get("dirichlet", {}).items():
            s.set_dirichlet(face, val)
        return s

    def close(self):
        if getattr(self, "h", None):
            self.lib.pmf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up ----------------------------------------------------------------
    def set_kappa(self, kx, ky=None, kz=None):
        px, dev, ka = _ptr(kx)
        py_, _, kb = _ptr(ky if ky is not None else kx)
        pz, _, kc = _ptr(kz if kz is not None else kx)
        _native.check(self.lib.pmf_set_kappa(self.h, px, py_, pz, dev))

    def set_dirichlet(self, face, value):
        f = FACE_IDS[face] if isinstance(face, str) else int(face)
        _native.check(self.lib.pmf_set_dirichlet(self.h, f, float(value)))

    def setup(self):
        _native.check(self.lib.pmf_setup(self.h))

    # -- vectors -----------------------------------------------------------------
    def _io(self, fn, x, out):
        px, dev, keep = _ptr(x)
        if out is None:
            if dev:
                import torch
                out = torch.empty_like(x)
            else:
                out = np.empty(self.n)
        po, dev2, keep2 = _ptr(out, writable=True)
        if dev != dev2:
            raise ValueError("input and output must both be host or both be device arrays")
        _native.check(fn(self.h, px, po, dev))
        return out

    def rhs(self, source, out=None):
        return self._io(self.lib.pmf_rhs, source, out)

    def apply_A(self, x, out=None):
        return self._io(self.lib.pmf_apply_A, x, out)

    def pc_apply(self, x, out=None):
        return self._io(self.lib.pmf_pc_apply, x, out)

    def solve(self, b, out=None):
        """PCG solve; returns (x, its, rnorm, reason)."""
        pb, dev, keep = _ptr(b)
        if out is None:
            if dev:
                import torch
                out = torch.empty_like(b)
            else:
                out = np.empty(self.n)
        px, dev2, keep2 = _ptr(out, writable=True)
        its = C.c_int(0)
        rn = C.c_double(0.0)
        reason = C.c_int(0)
        _native.check(self.lib.pmf_solve(self.h, pb, px, dev, C.byref(its), C.byref(rn), C.byref(reason)))
        return out, its.value, rn.value, REASONS.get(reason.value, str(reason.value))

    # -- introspection -----------------------------------------------------------
    def info(self):
        a = np.zeros(12, dtype=np.int32)
        _native.check(self.lib.pmf_get_info(self.h, a.ctypes.data_as(C.c_void_p)))
        keys = ("ncell", "nsub", "nrank", "spr", "kmax", "nr", "en2", "n3", "max_cells", "max_lines", "precision",
                "is_setup")
        return dict(zip(keys, (int(v) for v in a)))

    def eigen_lv1(self):
        inf = self.info()
        k = inf["kmax"]
        ev = np.zeros(inf["nsub"] * k)
        ks = np.zeros(inf["nsub"], dtype=np.int32)
        it = np.zeros(inf["nsub"], dtype=np.int32)
        stt = np.zeros(inf["nsub"], dtype=np.int32)
        _native.check(self.lib.pmf_get_eigen_lv1(self.h, ev.ctypes.data_as(C.c_void_p), ks.ctypes.data_as(C.c_void_p),
                                                 it.ctypes.data_as(C.c_void_p), stt.ctypes.data_as(C.c_void_p)))
        return ev.reshape(inf["nsub"], k), ks, it, stt

    def eigen_lv2(self):
        inf = self.info()
        ev = np.zeros(inf["nrank"] * inf["en2"])
        ks = np.zeros(inf["nrank"], dtype=np.int32)
        it = np.zeros(inf["nrank"], dtype=np.int32)
        _native.check(self.lib.pmf_get_eigen_lv2(self.h, ev.ctypes.data_as(C.c_void_p), ks.ctypes.data_as(C.c_void_p),
                                                 it.ctypes.data_as(C.c_void_p)))
        return ev.reshape(inf["nrank"], inf["en2"]), ks, it

    def subdomains(self):
        inf = self.info()
        b = np.zeros(inf["nsub"] * 6, dtype=np.int32)
        r = np.zeros(inf["nsub"], dtype=np.int32)
        _native.check(self.lib.pmf_get_subdomains(self.h, b.ctypes.data_as(C.c_void_p), r.ctypes.data_as(C.c_void_p)))
        return b.reshape(-1, 6), r

    def phi(self):
        inf = self.info()
        out = np.zeros(self.n * inf["kmax"])
        _native.check(self.lib.pmf_get_phi(self.h, out.ctypes.data_as(C.c_void_p)))
        return out.reshape(self.n, inf["kmax"])

    def coarse_blocks(self):
        inf = self.info()
        k = inf["kmax"]
        out = np.zeros(inf["nsub"] * 7 * k * k)
        _native.check(self.lib.pmf_get_coarse_blocks(self.h, out.ctypes.data_as(C.c_void_p)))
        return out.reshape(inf["nsub"], 7, k, k)

    def stages(self):
        t = np.zeros(10)
        _native.check(self.lib.pmf_get_stages(self.h, t.ctypes.data_as(C.c_void_p)))
        return dict(zip(STAGE_NAMES, t.tolist()))

    def timing(self):
        a, b = C.c_double(), C.c_double()
        _native.check(self.lib.pmf_get_timing(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def learned_stats(self):
        """Learned start of the last set-up: used (0/1), fallbacks, LOBPCG iterations from the
        learned start, iterations of the fallbacks, network inference ms."""
        st = (C.c_longlong * 4)()
        nm = C.c_double()
        _native.check(self.lib.pmf_get_learned_stats(self.h, st, C.byref(nm)))
        return {"used": int(st[0]), "fallbacks": int(st[1]), "learned_iters": int(st[2]),
                "fallback_iters": int(st[3]), "net_ms": float(nm.value)}

    PROFILE_CLASSES = ("lv1_first", "lv1_with_y", "resid_restrict", "coarse", "prolong", "cg_p_update_Ap",
                       "cg_x_r_update", "beta")

    def profile_iteration(self, reps=5):
        """Device ms per PCG iteration by kernel class and launch groups per iteration (see pmf_b200.h)."""
        ms = np.zeros(8)
        nl = np.zeros(8, dtype=np.int32)
        _native.check(self.lib.pmf_profile_iteration(self.h, int(reps), ms.ctypes.data_as(C.c_void_p),
                                                     nl.ctypes.data_as(C.c_void_p)))
        return {k: (float(m), int(n)) for k, m, n in zip(self.PROFILE_CLASSES, ms, nl)}


class BatchSolver(DarcySolver):
    """Independent problems set up and solved together (pmf_batch_*).

    ``problems``: problem dicts as made by ``premixfem_b200.fields`` (dom, mesh,
    kappa, dirichlet); ``sds``: subdomains per axis of each problem (one virtual
    rank per problem).  Vectors of the batch live on the shared mesh the
    library lays the problems out on; ``pack`` / ``unpack`` convert between it
    and per-problem arrays."""

    def __init__(self, problems, sds, options=""):
        self.lib = _native.load()
        self.nprob = len(problems)
        if isinstance(options, dict):
            options = options_string(options)
        self.options = options
        dom = np.ascontiguousarray([p["dom"] for p in problems], dtype=np.float64).ravel()
        mesh = np.ascontiguousarray([p["mesh"] for p in problems], dtype=np.int32).ravel()
        sd = np.ascontiguousarray(sds, dtype=np.int32).ravel()
        h = C.c_void_p()
        _native.check(self.lib.pmf_batch_create(self.nprob, dom.ctypes.data_as(C.c_void_p),
                                                mesh.ctypes.data_as(C.c_void_p), sd.ctypes.data_as(C.c_void_p),
                                                options.encode(), C.byref(h)))
        self.h = h
        shared = np.zeros(3, dtype=np.int32)
        z0 = np.zeros(self.nprob, dtype=np.int32)
        _native.check(self.lib.pmf_batch_info(self.h, shared.ctypes.data_as(C.c_void_p), z0.ctypes.data_as(C.c_void_p)))
        self.mesh = tuple(int(v) for v in shared)
        self.z0 = [int(v) for v in z0]
        self.meshes = [tuple(int(v) for v in p["mesh"]) for p in problems]
        self.n = self.mesh[0] * self.mesh[1] * self.mesh[2]
        for q, p in enumerate(problems):
            for face, v in p.get("dirichlet", {}).items():
                _native.check(self.lib.pmf_batch_set_dirichlet(self.h, q, FACE_IDS[face], float(v)))

    def pack(self, arrays):
        """Per-problem arrays (natural order, x fastest) -> one shared-mesh vector (float64, zero padding)."""
        M, N, P = self.mesh
        out = np.zeros((P, N, M))
        for q, a in enumerate(arrays):
            Mq, Nq, Pq = self.meshes[q]
            out[self.z0[q]:self.z0[q] + Pq, :Nq, :Mq] = np.asarray(a, dtype=np.float64).reshape(Pq, Nq, Mq)
        return out.ravel()

    def unpack(self, v):
        """One shared-mesh vector -> the per-problem arrays (flat, natural order)."""
        M, N, P = self.mesh
        v = np.asarray(v).reshape(P, N, M)
        return [np.ascontiguousarray(v[self.z0[q]:self.z0[q] + Pq, :Nq, :Mq]).ravel()
                for q, (Mq, Nq, Pq) in enumerate(self.meshes)]

    def set_kappa_problems(self, problems):
        self.set_kappa(*(self.pack([p["kappa"][d] for p in problems]) for d in range(3)))

    def set_dirichlet(self, face, value):
        raise ValueError("a batch takes its Dirichlet faces per problem (from the problem dicts)")

    def solve(self, b, out=None):
        """One PCG per problem; returns (x, its, rnorm, reasons), the last three one entry per problem."""
        pb, dev, keep = _ptr(b)
        if out is None:
            if dev:
                import torch
                out = torch.empty_like(b)
            else:
                out = np.empty(self.n)
        px, dev2, keep2 = _ptr(out, writable=True)
        its = np.zeros(self.nprob, dtype=np.int32)
        rn = np.zeros(self.nprob)
        reason = np.zeros(self.nprob, dtype=np.int32)
        _native.check(self.lib.pmf_batch_solve(self.h, pb, px, dev, its.ctypes.data_as(C.c_void_p),
                                               rn.ctypes.data_as(C.c_void_p), reason.ctypes.data_as(C.c_void_p)))
        return out, its, rn, [REASONS.get(int(r), str(int(r))) for r in reason]


# ---------------------------------------------------------------------------
# The reference's interface (src/PreMixFEM_3D.h:32-67), same names and order.
class PCCtx:
    """Mirror of the reference's PCCtx (src/PreMixFEM_3D.h:32-45)."""

    def __init__(self):
        self.solver = None
        self.kappa = [None, None, None]
        self.dirichlet = {}
        self.L = self.W = self.H = 0.0
        self.M = self.N = self.P = 0
        self.H_x = self.H_y = self.H_z = 0.0


def PC_init(s_ctx: PCCtx, dom, mesh, options=""):
    """PC_init (src/PreMixFEM_3D.c:1650-1741): checks dom/mesh, reads options."""
    s_ctx.solver = DarcySolver(dom, mesh, options)
    s_ctx.L, s_ctx.W, s_ctx.H = (float(v) for v in dom)
    s_ctx.M, s_ctx.N, s_ctx.P = (int(v) for v in mesh)
    s_ctx.H_x, s_ctx.H_y, s_ctx.H_z = s_ctx.L / s_ctx.M, s_ctx.W / s_ctx.N, s_ctx.H / s_ctx.P
    return 0


def PC_create_A(s_ctx: PCCtx):
    """PC_create_A (src/PreMixFEM_3D.c:1757-1824): returns the operator as a matvec callable."""
    s = s_ctx.solver
    s.set_kappa(*s_ctx.kappa)
    for f, v in s_ctx.dirichlet.items():
        s.set_dirichlet(f, v)
    return s.apply_A


def PC_setup(s_ctx: PCCtx):
    """PC_setup / _PC_setup (src/PreMixFEM_3D.c:1392-1427, 1826-1838)."""
    s_ctx.solver.setup()
    return 0


def PC_apply_vec(s_ctx: PCCtx, x, y=None):
    """PC_apply_vec (src/PreMixFEM_3D.c:1840-1936): y = B x (y is overwritten)."""
    return s_ctx.solver.pc_apply(x, y)


def PC_print_stat(s_ctx: PCCtx):
    """PC_print_stat (src/PreMixFEM_3D.c:1954-1999), single process."""
    s = s_ctx.solver
    ev1, ks, _, _ = s.eigen_lv1()
    ev2, ks2, _ = s.eigen_lv2()
    emax1 = np.array([ev1[i, ks[i] - 1] for i in range(len(ks))])
    st = s.stages()
    print(f"eigen_max_lv1_range=[{emax1.min():.5E}, {emax1.max():.5E}], \teigen_min_lv1_range=[{ev1[:, 0].min():.5E}, "
          f"{ev1[:, 0].max():.5E}], \teigen_num_lv1_range=[{ks.min()}, {ks.max()}].")
    emax2 = np.array([ev2[i, ks2[i] - 1] for i in range(len(ks2))])
    print(f"eigen_max_lv2_range=[{emax2.min():.5E}, {emax2.max():.5E}], \teigen_min_lv2_range=[{ev2[:, 0].min():.5E}, "
          f"{ev2[:, 0].max():.5E}], \teigen_num_lv2_range=[{ks2.min()}, {ks2.max()}], \tsize_mat_lv3={int(ks2.sum())}.")
    print(", \t".join(f"{k}=[{v:.5f}, {v:.5f}]" for k, v in st.items()) + ".")
    return 0


def PC_final(s_ctx: PCCtx):
    """PC_final / PC_final_default (src/PreMixFEM_3D.c:2001-2046)."""
    if s_ctx.solver is not None:
        s_ctx.solver.close()
        s_ctx.solver = None
    return 0
