"""CPU FP64 oracle for the three-level GMsFEM-preconditioned CG path.

TEST INFRASTRUCTURE ONLY.  This is a plain numpy/scipy restatement of the
reference's preconditioner (src/PreMixFEM_3D.c of Laphet/PreMixFEM) and of the
PETSc KSPCG loop the reference drives it with.  Only tests/, the smoke check
and the CPU-baseline leg of bench.py may import it; the product path (the
CUDA library under premixfem_b200/) never calls it.

PARITY UNPINNED.  The reference ships no tests, fixtures or golden vectors,
and it cannot be compiled here (it needs PETSc, SLEPc, MPI, MUMPS and
SuperLU_dist, none of which are installed).  This oracle is therefore pinned
only to mathematics: tests/test_oracle.py checks it against closed-form
eigenvalues of constant-coefficient operators, exact Cholesky on chains, the
textbook IC(0) definition and direct sparse solves.  tests/golden/ holds its
own results on the reference's test.c and cross-field problems: they pin the
oracle against its own changes, not against the reference.

Third-party arithmetic restated here (pinned versions from the reference's
build notes, Compiling_optimized_PETSc_for_AMD_CPUs.md:76-83):
  * SLEPc (slepc-3811 tarball) EPS Krylov-Schur with shift-and-invert, target
    -1e-12 -> dense ``scipy.linalg.eigh`` on the same GHEP / HEP.  Generalized
    eigenvectors come back B-normalised (v^T M v = 1), the normalisation SLEPc
    documents for GHEP; standard ones are 2-norm normalised.
  * PETSc PCICC (level 0, natural ordering; SBAIJ) -> IC(0) on the 7-point
    pattern, solved with sparse triangular solves.
  * MUMPS 5.5.1 Cholesky / SuperLU_dist 8.1.2 LU on the coarse matrices ->
    dense Cholesky (``chol_semidef`` below; pivots below a relative threshold
    are treated as null directions, which only matters for the singular
    coarse matrices of pure-Neumann problems).
  * PETSc KSPCG with KSP_NORM_UNPRECONDITIONED -> ``pcg`` below, same
    recurrences and the KSPConvergedDefault test ||r_k|| <= rtol*||r_0||.

Extensions beyond the reference (flagged, used by the benchmark fields):
  * Dirichlet faces: a boundary transmissibility t_b = |f|^2/|K| * 2*k_cell
    is added to the diagonal of A and therefore of every level's local and
    Galerkin matrix (the way src/spe10.c:783,925,1009,1127,1286,1517 folds its
    well term into all levels).  In the MOD mass matrix the face adds 2*t_b
    (the MOD weight of any face is twice its transmissibility); DIAG picks it
    up through diag(A_i); MEAN ignores it.
  * Virtual ranks: the reference's DMDA process grid (px, py, pz) is given
    explicitly, so one process reproduces a multi-rank run; per-axis
    subdomain counts ``sd=(sx, sy, sz)`` per rank.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

NIL = 1.0e-12  # src/PreMixFEM_3D.h:15
EIG_OP_MOD, EIG_OP_MEAN, EIG_OP_DIAG = 0, 1, 2  # src/PreMixFEM_3D.h:28-30


@dataclass
class Options:
    """Preconditioner options; names follow PC_init (src/PreMixFEM_3D.c:1662-1705)."""

    sd: tuple = (2, 2, 2)
    vranks: tuple = (1, 1, 1)
    en_lv1: int = 4
    en_lv2: int = 4
    eb_lv1: float = -1.0
    eb_lv2: float = -1.0
    si_lv1: int = 1
    si_lv2: int = 1
    eg_op: int = EIG_OP_MOD
    use_W_cycle: bool = False
    no_shift_A_cc: bool = False
    use_full_Cholesky_lv1: bool = False
    use_2level: bool = False
    rtol: float = 1.0e-8
    max_it: int = 10000
    # -ksp_constant_null_space (PETSc KSPSetFromOptions, read by the drivers'
    # KSPSetFromOptions call, src/Expe_scal.c:115): the constant vector is the
    # operator's null space, removed from every preconditioned residual
    constant_null_space: bool = False
    # store the local eigenvectors rounded to FP32, as the mixed form keeps the
    # coarse basis (the Galerkin products and solves stay FP64)
    phi_fp32: bool = False
    eig_method: str = "dense"  # "dense": scipy.linalg.eigh; "arpack": eigsh shift-and-invert (SLEPc-like)

    def normalized(self):
        o = Options(**self.__dict__)
        sd = o.sd
        if isinstance(sd, int):
            sd = (sd, sd, sd)
            # src/PreMixFEM_3D.c:1718-1721: a single subdomain is reset to 2.
            if sd[0] == 1:
                sd = (2, 2, 2)
        o.sd = tuple(int(v) for v in sd)
        o.vranks = tuple(int(v) for v in o.vranks)
        o.si_lv1 = max(1, int(o.si_lv1))  # :1664
        o.si_lv2 = max(1, int(o.si_lv2))  # :1668
        o.eb_lv1 = 1.0 / NIL if o.eb_lv1 < 0.0 else o.eb_lv1  # :1689
        o.eb_lv2 = 1.0 / NIL if o.eb_lv2 < 0.0 else o.eb_lv2  # :1693
        return o


def split(n, parts):
    """Near-equal split, first n % parts pieces one longer.

    src/PreMixFEM_3D.c:62-71 (_PC_setup_lv1_partition); the same rule gives the
    DMDA ownership ranges of a PETSC_DECIDE process grid.
    """
    lens = [n // parts + (1 if (n % parts) > i else 0) for i in range(parts)]
    starts = [0] * parts
    for i in range(1, parts):
        starts[i] = starts[i - 1] + lens[i - 1]
    return starts, lens


@dataclass
class Layout:
    """Virtual-rank boxes and their subdomains, in global dof order.

    Ranks are ordered x-fastest (PETSc DMDA rank order); inside a rank the
    coarse elements are ordered x-fastest (src/PreMixFEM_3D.c:23-27).
    """

    mesh: tuple
    ranks: list = field(default_factory=list)  # (x0, nx, y0, ny, z0, nz)
    subs: list = field(default_factory=list)  # (x0, nx, y0, ny, z0, nz, rank)
    subs_per_rank: int = 0

    @staticmethod
    def build(mesh, vranks, sd):
        M, N, P = mesh
        px, py, pz = vranks
        rx = split(M, px)
        ry = split(N, py)
        rz = split(P, pz)
        lay = Layout(mesh=tuple(mesh))
        for kz in range(pz):
            for ky in range(py):
                for kx in range(px):
                    box = (rx[0][kx], rx[1][kx], ry[0][ky], ry[1][ky], rz[0][kz], rz[1][kz])
                    r = len(lay.ranks)
                    lay.ranks.append(box)
                    sx = split(box[1], sd[0])
                    sy = split(box[3], sd[1])
                    sz = split(box[5], sd[2])
                    for cz in range(sd[2]):
                        for cy in range(sd[1]):
                            for cx in range(sd[0]):
                                lay.subs.append((box[0] + sx[0][cx], sx[1][cx], box[2] + sy[0][cy], sy[1][cy],
                                                 box[4] + sz[0][cz], sz[1][cz], r))
        lay.subs_per_rank = sd[0] * sd[1] * sd[2]
        for s in lay.subs:
            if min(s[1], s[3], s[5]) < 1:
                raise ValueError("empty subdomain: too many subdomains for the mesh")
        return lay


def box_cells(mesh, box):
    """Flat natural-order cell ids of a box, local x-fastest ordering."""
    M, N, P = mesh
    x0, nx, y0, ny, z0, nz = box[:6]
    z = np.arange(z0, z0 + nz)[:, None, None]
    y = np.arange(y0, y0 + ny)[None, :, None]
    x = np.arange(x0, x0 + nx)[None, None, :]
    return ((z * N + y) * M + x).ravel()


class Operator:
    """Cell-centred 7-point TPFA operator of PC_create_A (src/PreMixFEM_3D.c:1757-1824)."""

    def __init__(self, problem):
        self.problem = problem
        M, N, P = self.mesh = problem["mesh"]
        L, W, H = problem["dom"]
        self.H = (L / M, W / N, H / P)  # :1707-1709
        Hx, Hy, Hz = self.H
        meas_elem = Hx * Hy * Hz  # _PC_setup :1403-1406
        f_yz, f_zx, f_xy = Hy * Hz, Hz * Hx, Hx * Hy
        self.meas_elem = meas_elem
        # meas_face * meas_face / meas_elem, evaluated left to right as in the reference
        self.cx = f_yz * f_yz / meas_elem
        self.cy = f_zx * f_zx / meas_elem
        self.cz = f_xy * f_xy / meas_elem
        kx, ky, kz = problem["kappa"]
        self.kappa = (kx, ky, kz)
        shape = (P, N, M)
        tx = np.zeros(shape)
        ty = np.zeros(shape)
        tz = np.zeros(shape)
        # harmonic mean 2/(1/k_L + 1/k_R), :1787, :1798, :1809
        tx[:, :, 1:] = self.cx * (2.0 / (1.0 / kx[:, :, :-1] + 1.0 / kx[:, :, 1:]))
        ty[:, 1:, :] = self.cy * (2.0 / (1.0 / ky[:, :-1, :] + 1.0 / ky[:, 1:, :]))
        tz[1:, :, :] = self.cz * (2.0 / (1.0 / kz[:-1, :, :] + 1.0 / kz[1:, :, :]))
        self.tx, self.ty, self.tz = tx, ty, tz
        # Dirichlet extension: t_b = c * 2 k_cell on the diagonal, t_b * p_D on the rhs.
        db = np.zeros(shape)
        bval = np.zeros(shape)
        self.dir_faces = {}
        for face, val in problem.get("dirichlet", {}).items():
            if face == "x-":
                tb = self.cx * (2.0 * kx[:, :, 0]); sl = (slice(None), slice(None), 0)
            elif face == "x+":
                tb = self.cx * (2.0 * kx[:, :, M - 1]); sl = (slice(None), slice(None), M - 1)
            elif face == "y-":
                tb = self.cy * (2.0 * ky[:, 0, :]); sl = (slice(None), 0, slice(None))
            elif face == "y+":
                tb = self.cy * (2.0 * ky[:, N - 1, :]); sl = (slice(None), N - 1, slice(None))
            elif face == "z-":
                tb = self.cz * (2.0 * kz[0, :, :]); sl = (0, slice(None), slice(None))
            elif face == "z+":
                tb = self.cz * (2.0 * kz[P - 1, :, :]); sl = (P - 1, slice(None), slice(None))
            else:
                raise ValueError(face)
            db[sl] += tb
            bval[sl] += tb * val
            self.dir_faces[face] = val
        self.db = db
        self.bval = bval
        # Diagonal accumulated in the order PETSc's ADD_VALUES assembly sees it:
        # own left/down/back faces, then the faces added by the +x, +y, +z neighbours.
        d = tx + ty
        d = d + tz
        d[:, :, :-1] += tx[:, :, 1:]
        d[:, :-1, :] += ty[:, 1:, :]
        d[:-1, :, :] += tz[1:, :, :]
        d = d + db
        self.diag = d
        n = M * N * P
        self.n = n
        txf, tyf, tzf = tx.ravel(), ty.ravel(), tz.ravel()
        rows = [np.arange(n)]
        cols = [np.arange(n)]
        vals = [d.ravel()]
        for tf, off in ((txf, 1), (tyf, M), (tzf, M * N)):
            c = np.nonzero(tf)[0]
            rows += [c, c - off]
            cols += [c - off, c]
            vals += [-tf[c], -tf[c]]
        self.A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))

    def rhs(self):
        return (self.problem["source"] + self.bval).ravel().copy()

    def matvec(self, x):
        return self.A @ x

    def crossing(self, box):
        """Per-cell sum of transmissibilities of faces leaving ``box`` into the domain."""
        M, N, P = self.mesh
        x0, nx, y0, ny, z0, nz = box[:6]
        out = np.zeros((nz, ny, nx))
        zs, ys, xs = slice(z0, z0 + nz), slice(y0, y0 + ny), slice(x0, x0 + nx)
        if x0 > 0:
            out[:, :, 0] += self.tx[zs, ys, x0]
        if x0 + nx < M:
            out[:, :, nx - 1] += self.tx[zs, ys, x0 + nx]
        if y0 > 0:
            out[:, 0, :] += self.ty[zs, y0, xs]
        if y0 + ny < N:
            out[:, ny - 1, :] += self.ty[zs, y0 + ny, xs]
        if z0 > 0:
            out[0, :, :] += self.tz[z0, ys, xs]
        if z0 + nz < P:
            out[nz - 1, :, :] += self.tz[z0 + nz, ys, xs]
        return out.ravel()

    def principal(self, box):
        """Principal submatrix of A on a box: the level-1 local matrix (:93-196)."""
        idx = box_cells(self.mesh, box)
        return self.A[idx][:, idx].tocsr()

    def neumann(self, box):
        """A restricted to a box with no-flux on the box faces (:245-320, :938-1076)."""
        Ab = self.principal(box)
        return (Ab - sp.diags(self.crossing(box))).tocsr()

    def mass_diag(self, box, eg_op):
        """Diagonal M_i of the level-2 GHEP (src/PreMixFEM_3D.c:243-346).

        EIG_OP_MOD reproduces the reference's x-direction accumulation: the
        face between local cells lx-1 and lx is added to cell lx-1 (:266), so a
        cell gets its right face twice when it is not the last in its row and
        its left face only when it is the first (:271-274).
        """
        M, N, P = self.mesh
        Hx, Hy, Hz = self.H
        kx, ky, kz = self.kappa
        x0, nx, y0, ny, z0, nz = box[:6]
        if eg_op == EIG_OP_MEAN:
            sl = (slice(z0, z0 + nz), slice(y0, y0 + ny), slice(x0, x0 + nx))
            return (kx[sl] + ky[sl] + kz[sl]).ravel()  # :332-333
        if eg_op == EIG_OP_DIAG:
            return self.neumann(box).diagonal().copy()
        out = np.zeros((nz, ny, nx))

        def avg(k, a, b):
            return 2.0 / (1.0 / k[a] + 1.0 / k[b])

        for lz in range(nz):
            ez = z0 + lz
            for ly in range(ny):
                ey = y0 + ly
                for lx in range(nx):
                    ex = x0 + lx
                    if lx >= 1:
                        out[lz, ly, lx - 1] += 2.0 * avg(kx, (ez, ey, ex - 1), (ez, ey, ex)) / Hx / Hx
                    elif ex >= 1:
                        out[lz, ly, lx] += 2.0 * avg(kx, (ez, ey, ex - 1), (ez, ey, ex)) / Hx / Hx
                    if ex + 1 != M:
                        out[lz, ly, lx] += 2.0 * avg(kx, (ez, ey, ex), (ez, ey, ex + 1)) / Hx / Hx
                    if ey >= 1:
                        out[lz, ly, lx] += 2.0 * avg(ky, (ez, ey - 1, ex), (ez, ey, ex)) / Hy / Hy
                    if ey + 1 != N:
                        out[lz, ly, lx] += 2.0 * avg(ky, (ez, ey, ex), (ez, ey + 1, ex)) / Hy / Hy
                    if ez >= 1:
                        out[lz, ly, lx] += 2.0 * avg(kz, (ez - 1, ey, ex), (ez, ey, ex)) / Hz / Hz
                    if ez + 1 != P:
                        out[lz, ly, lx] += 2.0 * avg(kz, (ez, ey, ex), (ez + 1, ey, ex)) / Hz / Hz
        # Dirichlet extension: 2 t_b per boundary face, written as 2*(2k)/H^2 before the |K| scaling.
        for face in self.dir_faces:
            if face == "x-" and x0 == 0:
                out[:, :, 0] += 2.0 * (2.0 * kx[z0:z0 + nz, y0:y0 + ny, 0]) / Hx / Hx
            if face == "x+" and x0 + nx == M:
                out[:, :, nx - 1] += 2.0 * (2.0 * kx[z0:z0 + nz, y0:y0 + ny, M - 1]) / Hx / Hx
            if face == "y-" and y0 == 0:
                out[:, 0, :] += 2.0 * (2.0 * ky[z0:z0 + nz, 0, x0:x0 + nx]) / Hy / Hy
            if face == "y+" and y0 + ny == N:
                out[:, ny - 1, :] += 2.0 * (2.0 * ky[z0:z0 + nz, N - 1, x0:x0 + nx]) / Hy / Hy
            if face == "z-" and z0 == 0:
                out[0, :, :] += 2.0 * (2.0 * kz[0, y0:y0 + ny, x0:x0 + nx]) / Hz / Hz
            if face == "z+" and z0 + nz == P:
                out[nz - 1, :, :] += 2.0 * (2.0 * kz[P - 1, y0:y0 + ny, x0:x0 + nx]) / Hz / Hz
        return (out * self.meas_elem).ravel()  # VecScale(diag_M_i, meas_elem), :343


def ic0_pivots(Aloc):
    """IC(0) pivots of a 7-point matrix in natural order.

    For the 7-point pattern no product L_ik L_jk survives the zero-fill rule,
    so IC(0) reduces to D_i = a_ii - sum_{j<i, a_ij != 0} a_ij^2 / D_j and the
    factor is (D + L) D^-1 (D + L^T), L = strict lower part of A.
    tests/test_oracle.py checks this against the general IC(0) definition.
    """
    A = sp.csr_matrix(Aloc)
    n = A.shape[0]
    D = np.zeros(n)
    indptr, indices, data = A.indptr, A.indices, A.data
    for i in range(n):
        s = 0.0
        aii = 0.0
        for p in range(indptr[i], indptr[i + 1]):
            j = indices[p]
            if j < i:
                s += data[p] * data[p] / D[j]
            elif j == i:
                aii = data[p]
        D[i] = aii - s
        if D[i] <= 0.0:
            raise FloatingPointError("non-positive IC(0) pivot")
    return D


def ic0_general(Adense):
    """Textbook IC(0) (lower factor restricted to the pattern of tril(A))."""
    A = np.asarray(Adense, dtype=np.float64)
    n = A.shape[0]
    L = np.zeros_like(A)
    pat = A != 0.0
    for j in range(n):
        L[j, j] = np.sqrt(A[j, j] - np.dot(L[j, :j], L[j, :j]))
        for i in range(j + 1, n):
            if pat[i, j]:
                L[i, j] = (A[i, j] - np.dot(L[i, :j], L[j, :j])) / L[j, j]
    return L


class IC0Solver:
    """Level-1 local solve (LL^T)^-1 with PCICC (src/PreMixFEM_3D.c:200-215)."""

    def __init__(self, Aloc):
        A = sp.csr_matrix(Aloc)
        self.D = ic0_pivots(A)
        Lo = sp.tril(A, k=-1).tocsr()
        self.lower = (Lo + sp.diags(self.D)).tocsr()
        self.upper = (Lo.T + sp.diags(self.D)).tocsr()

    def solve(self, r):
        u = spla.spsolve_triangular(self.lower, r, lower=True)
        return spla.spsolve_triangular(self.upper, self.D * u, lower=False)


class CholSolver:
    """Exact local Cholesky (-use_full_Cholesky_lv1, :205-207)."""

    def __init__(self, Aloc):
        self.c = sla.cho_factor(Aloc.toarray() if sp.issparse(Aloc) else Aloc)

    def solve(self, r):
        return sla.cho_solve(self.c, r)


def chol_semidef(A, rel_tol=1.0e-14):
    """Dense Cholesky tolerant of null directions.

    Returns (L, null) with L lower triangular; a pivot below rel_tol * max
    diagonal marks its column as a null direction (L column zeroed, pivot 1).
    For SPD inputs this is the ordinary Cholesky factor.
    """
    A = np.array(A, dtype=np.float64, copy=True)
    n = A.shape[0]
    scale = max(np.max(np.abs(np.diag(A))), 1e-300)
    if n > 2048:
        # large matrices: LAPACK's Cholesky, which is the loop below whenever no
        # pivot falls to the null threshold (checked on the computed pivots)
        try:
            Lf = sla.cholesky(A, lower=True, check_finite=False)
            if np.all(np.diag(Lf) ** 2 > rel_tol * scale):
                return Lf, np.zeros(n, dtype=bool)
        except sla.LinAlgError:
            pass
    L = np.zeros_like(A)
    null = np.zeros(n, dtype=bool)
    for j in range(n):
        d = A[j, j] - np.dot(L[j, :j], L[j, :j])
        if d <= rel_tol * scale:
            null[j] = True
            L[j, j] = 1.0
            continue
        L[j, j] = np.sqrt(d)
        L[j + 1:, j] = (A[j + 1:, j] - L[j + 1:, :j] @ L[j, :j]) / L[j, j]
    return L, null


def chol_semidef_solve(Lnull, b):
    L, null = Lnull
    y = sla.solve_triangular(L, b, lower=True)
    y[null] = 0.0
    x = sla.solve_triangular(L.T, y, lower=False)
    x[null] = 0.0
    return x


def local_basis(op: Operator, box, o: Options):
    """One subdomain's level-2 basis (_PC_setup_lv2_eigen, :224-421): the
    en_lv1 smallest pairs of A_i^N v = lambda M_i v and the adaptive count
    (:369-383).  ``o`` must be normalised.  Returns (w, V, num, vmax)."""
    k = o.en_lv1
    An = op.neumann(box)
    An = An if o.eig_method == "arpack" else An.toarray()
    Md = op.mass_diag(box, o.eg_op)
    if k > An.shape[0]:
        raise ValueError("en_lv1 larger than a subdomain")
    if o.eig_method == "arpack" and k < An.shape[0] - 1:
        # SLEPc EPS with STSINVERT and target -NIL (:354-365): Lanczos on (A + NIL M)^-1 M
        w, V = spla.eigsh(sp.csc_matrix(An), k=k, M=sp.diags(Md).tocsc(), sigma=-NIL, which="LM")
        order = np.argsort(w)
        w, V = w[order], V[:, order]
    else:
        w, V = sla.eigh(An, np.diag(Md), subset_by_index=[0, k - 1])
    if o.phi_fp32:
        V = V.astype(np.float32).astype(np.float64)
    num, vmax = k, w[k - 1]
    for j in range(k):
        if w[j] >= o.eb_lv1:
            num, vmax = j + 1, w[j]
            break
    return w, V, num, vmax


def level3_basis(AN, o: Options):
    """One virtual rank's level-3 vectors (_PC_setup_lv3_eigen, :1086-1115):
    the en_lv2 smallest eigenpairs of its rank-Neumann coarse matrix and the
    adaptive count.  Returns (w, V[:, :num], num, vmax)."""
    AN = AN.toarray() if sp.issparse(AN) else np.asarray(AN)
    k = min(o.en_lv2, AN.shape[0])
    w, V = sla.eigh(AN, subset_by_index=[0, k - 1])
    num, vmax = k, w[k - 1]
    for j in range(k):
        if w[j] >= o.eb_lv2:
            num, vmax = j + 1, w[j]
            break
    return w, V[:, :num], num, vmax


def cycle_schedule(o: Options):
    """The visits of PC_apply_vec (:1840-1936) for normalised options: levels
    1, 2, 3 or "2g" (the 2-level branch's global coarse solve)."""
    s1 = [1] * o.si_lv1
    s2 = [2] * o.si_lv2
    if o.use_W_cycle and not o.use_2level:  # :1857-1894
        return s1 + s2 + [3] + s2 + [3] + s2 + s1
    if o.use_2level:  # :1918-1922
        return s1 + ["2g"] + s1
    return s1 + s2 + [3] + s2 + s1  # :1896-1928


class Preconditioner:
    """The three-level preconditioner: _PC_setup (:1392-1427) + PC_apply_vec (:1840-1936)."""

    def __init__(self, op: Operator, opts: Options):
        self.op = op
        self.opts = o = opts.normalized()
        self.lay = Layout.build(op.mesh, o.vranks, o.sd)
        self.stats = {}
        self._setup_lv1()
        self._setup_lv2_eigen()
        if o.use_2level:
            self._setup_lv2_c()
        else:
            self._setup_lv2_J()
            self._setup_lv3_eigen()
            self._setup_lv3_cc()

    # level 1 -----------------------------------------------------------
    def _setup_lv1(self):
        self.sub_idx = []
        self.lv1 = []
        for s in self.lay.subs:
            idx = box_cells(self.op.mesh, s)
            self.sub_idx.append(idx)
            Aloc = self.op.principal(s)
            self.lv1.append(CholSolver(Aloc) if self.opts.use_full_Cholesky_lv1 else IC0Solver(Aloc))

    def apply_lv1(self, r):
        """_PC_apply_vec_lv1 (:1429-1479): additive block solves."""
        y = np.zeros_like(r)
        for idx, sol in zip(self.sub_idx, self.lv1):
            y[idx] += sol.solve(r[idx])
        return y

    # level 2 eigen -----------------------------------------------------
    def _setup_lv2_eigen(self):
        o = self.opts
        self.eig_num_lv1 = []
        self.eig_min_lv1 = []
        self.eig_max_lv1 = []
        self.eigvals_lv1 = []
        self.phi = []  # per subdomain (n_s, en_lv1) M-normalised eigenvectors
        for s in self.lay.subs:
            w, V, num, vmax = local_basis(self.op, s, o)
            self.eigvals_lv1.append(w)
            self.eig_num_lv1.append(num)
            self.eig_min_lv1.append(w[0])
            self.eig_max_lv1.append(vmax)
            self.phi.append(V)
        self.dof_idx = np.concatenate([[0], np.cumsum(self.eig_num_lv1)])
        n, nc = self.op.n, int(self.dof_idx[-1])
        rows, cols, vals = [], [], []
        for si, (idx, V) in enumerate(zip(self.sub_idx, self.phi)):
            for j in range(self.eig_num_lv1[si]):
                rows.append(idx)
                cols.append(np.full(idx.size, self.dof_idx[si] + j))
                vals.append(V[:, j])
        self.Phi = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, nc))
        self.A2full = (self.Phi.T @ self.op.A @ self.Phi).toarray()

    def rank_dofs(self, r):
        spr = self.lay.subs_per_rank
        return np.arange(self.dof_idx[r * spr], self.dof_idx[(r + 1) * spr])

    def _setup_lv2_J(self):
        """_PC_setup_lv2_J (:737-916): per-rank principal block of Phi^T A Phi, Cholesky."""
        self.lv2 = []
        for r in range(len(self.lay.ranks)):
            d = self.rank_dofs(r)
            self.lv2.append((d, chol_semidef(self.A2full[np.ix_(d, d)])))

    def apply_lv2(self, r):
        """_PC_apply_vec_lv2 (:1539-1595)."""
        c = self.Phi.T @ r
        z = np.zeros_like(c)
        for d, f in self.lv2:
            z[d] = chol_semidef_solve(f, c[d])
        return self.Phi @ z

    def _setup_lv2_c(self):
        """_PC_setup_lv2_c (:423-735): global Phi^T A Phi (+NIL), direct solve."""
        Ac = self.A2full.copy()
        if not self.opts.no_shift_A_cc:
            Ac += NIL * np.eye(Ac.shape[0])
        self.lv2c = chol_semidef(Ac)

    def apply_lv2_2level(self, r):
        """_PC_apply_vec_lv2_2level (:1481-1537)."""
        return self.Phi @ chol_semidef_solve(self.lv2c, self.Phi.T @ r)

    # level 3 -------------------------------------------------------------
    def _setup_lv3_eigen(self):
        """_PC_setup_lv3_eigen (:918-1175): per-rank HEP on the rank-Neumann coarse matrix."""
        o = self.opts
        self.eig_num_lv2 = []
        self.eig_min_lv2 = []
        self.eig_max_lv2 = []
        self.eigvals_lv2 = []
        self.V3 = []
        psi_cols = []
        for r, box in enumerate(self.lay.ranks):
            d = self.rank_dofs(r)
            cells = box_cells(self.op.mesh, box)
            PhiR = self.Phi[cells][:, d]
            w, V, num, vmax = level3_basis(PhiR.T @ self.op.neumann(box) @ PhiR, o)
            self.eigvals_lv2.append(w)
            self.eig_num_lv2.append(num)
            self.eig_min_lv2.append(w[0])
            self.eig_max_lv2.append(vmax)
            self.V3.append((d, V))
            for j in range(num):
                col = np.zeros(self.Phi.shape[1])
                col[d] = V[:, j]
                psi_cols.append(col)
        self.Vmat = np.stack(psi_cols, axis=1)  # coarse-dof coefficients of Psi
        self.Psi = self.Phi @ self.Vmat

    def _setup_lv3_cc(self):
        """_PC_setup_lv3_cc (:1177-1390): Psi^T A Psi (+NIL), direct solve."""
        A3 = self.Vmat.T @ self.A2full @ self.Vmat
        if not self.opts.no_shift_A_cc:
            A3 = A3 + NIL * np.eye(A3.shape[0])  # :1361-1363
        self.A3 = A3
        self.lv3 = chol_semidef(A3)

    def apply_lv3(self, r):
        """_PC_apply_vec_lv3 (:1597-1648)."""
        return self.Psi @ chol_semidef_solve(self.lv3, self.Psi.T @ r)

    # cycle ------------------------------------------------------------------
    def schedule(self):
        return cycle_schedule(self.opts)

    def apply(self, x):
        """PC_apply_vec: y = 0, then r = x - A y; y += B_l r for each visit."""
        y = np.zeros_like(x)
        for lvl in self.schedule():
            r = x - self.op.A @ y
            if lvl == 1:
                y += self.apply_lv1(r)
            elif lvl == 2:
                y += self.apply_lv2(r)
            elif lvl == 3:
                y += self.apply_lv3(r)
            else:
                y += self.apply_lv2_2level(r)
        return y


def remove_constant(z):
    """MatNullSpaceRemove of a constant null space: z <- z - (sum z / n) 1."""
    return z - z.sum() / z.size


def pcg(A, b, apply_pc, rtol=1.0e-8, max_it=10000, abstol=1.0e-50, null_space=False):
    """PETSc KSPSolve_CG with KSP_NORM_UNPRECONDITIONED and KSPConvergedDefault.

    Returns (x, its, history, reason).  Convergence when ||r_k|| <= max(rtol
    ||r_0||, abstol) with r_0 = b (zero initial guess).  With ``null_space``
    (a constant null space attached to the operator) every preconditioned
    residual loses its mean, as KSP_PCApply does for a left preconditioner;
    b is not projected (the operator carries no transpose null space).
    """
    if null_space:
        inner = apply_pc

        def apply_pc(r):
            return remove_constant(inner(r))
    x = np.zeros_like(b)
    r = b.copy()
    dp = float(np.linalg.norm(r))
    hist = [dp]
    ttol = max(rtol * dp, abstol)
    if dp <= ttol:
        return x, 0, hist, "converged_atol"
    z = apply_pc(r)
    beta = float(z @ r)
    p = None
    betaold = dpi = 0.0
    i = 0
    its = 0
    while i < max_it:
        its = i + 1
        if beta == 0.0:
            return x, its, hist, "converged_atol"
        if i == 0:
            p = z.copy()
        else:
            p = z + (beta / betaold) * p
        dpiold = dpi
        w = A @ p
        dpi = float(p @ w)
        betaold = beta
        if dpi == 0.0 or (i > 0 and np.sign(dpi) * np.sign(dpiold) < 0):
            return x, its, hist, "diverged_indefinite"
        a = beta / dpi
        x += a * p
        r -= a * w
        dp = float(np.linalg.norm(r))
        hist.append(dp)
        if not np.isfinite(dp):
            return x, its, hist, "diverged_nanorinf"
        if dp <= ttol:
            return x, its, hist, "converged_rtol"
        z = apply_pc(r)
        beta = float(z @ r)
        i += 1
    return x, its, hist, "diverged_its"


def direct_solve(op: Operator, b):
    """FP64 direct solve; pure-Neumann problems get a zero-mean constraint."""
    if not op.dir_faces:
        n = op.n
        one = sp.csr_matrix(np.ones((n, 1)))
        K = sp.bmat([[op.A, one], [one.T, None]]).tocsc()
        sol = spla.spsolve(K, np.concatenate([b - b.mean(), [0.0]]))
        return sol[:n]
    return spla.spsolve(op.A.tocsc(), b)


def solve(problem, opts: Options):
    """Operator + preconditioner setup + PCG, returning a result dict."""
    op = Operator(problem)
    b = op.rhs()
    pc = Preconditioner(op, opts)
    x, its, hist, reason = pcg(op.A, b, pc.apply, rtol=pc.opts.rtol, max_it=pc.opts.max_it,
                               null_space=pc.opts.constant_null_space)
    return {"op": op, "pc": pc, "b": b, "x": x, "its": its, "hist": hist, "reason": reason}


def crop_around(problem, box):
    """The problem restricted to ``box`` plus a one-cell halo where the mesh has
    cells, and the box in the crop's coordinates.

    A subdomain's level-2 GHEP (src/PreMixFEM_3D.c:243-346) reads the
    permeability of its own cells and of their face neighbours, the global
    boundary flags of its cells and the Dirichlet faces it touches; the crop
    keeps all of them (a crop face that is not a global face is never reached
    from inside the box), so the local matrices are the same as on the full
    mesh without assembling the whole operator.
    """
    M, N, P = problem["mesh"]
    L, W, H = problem["dom"]
    h = (L / M, W / N, H / P)
    x0, nx, y0, ny, z0, nz = (int(v) for v in box[:6])
    lo = (max(0, x0 - 1), max(0, y0 - 1), max(0, z0 - 1))
    hi = (min(M, x0 + nx + 1), min(N, y0 + ny + 1), min(P, z0 + nz + 1))
    sl = (slice(lo[2], hi[2]), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
    mesh = (hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2])
    kap = tuple(np.ascontiguousarray(np.asarray(k)[sl]) for k in problem["kappa"])
    on = {"x-": lo[0] == 0, "x+": hi[0] == M, "y-": lo[1] == 0, "y+": hi[1] == N, "z-": lo[2] == 0, "z+": hi[2] == P}
    dirichlet = {f: v for f, v in problem.get("dirichlet", {}).items() if on[f]}
    crop = dict(mesh=mesh, dom=(h[0] * mesh[0], h[1] * mesh[1], h[2] * mesh[2]), kappa=kap,
                source=np.zeros((mesh[2], mesh[1], mesh[0])), dirichlet=dirichlet)
    return crop, (x0 - lo[0], nx, y0 - lo[1], ny, z0 - lo[2], nz)


def local_eigenvalues(problem, boxes, k, eg_op=EIG_OP_MOD, method="arpack"):
    """The k smallest eigenvalues of each subdomain's GHEP A_i^N v = lambda M_i v
    (src/PreMixFEM_3D.c:224-390), one row per box: dense ``eigh`` or ARPACK
    shift-and-invert with SLEPc's target -NIL (:354-365), computed on
    ``crop_around`` crops."""
    out = []
    for box in boxes:
        crop, cb = crop_around(problem, box)
        op = Operator(crop)
        An = op.neumann(cb)
        Md = op.mass_diag(cb, eg_op)
        if method == "arpack" and k < An.shape[0] - 1:
            w = spla.eigsh(sp.csc_matrix(An), k=k, M=sp.diags(Md).tocsc(), sigma=-NIL, which="LM",
                           return_eigenvectors=False, tol=0.0)
            w = np.sort(w)
        else:
            w = sla.eigh(An.toarray(), np.diag(Md), subset_by_index=[0, k - 1], eigvals_only=True)
        out.append(w)
    return np.array(out)


def eigenvalue_errors(ev, ref):
    """Relative errors of computed local eigenvalues ``ev`` against ``ref``
    (rows: subdomains).  Returns (max relative error over the eigenvalues
    above 1e-8 x the row's largest, max |error| / row's largest over the
    others, i.e. the near-zero modes such as the constant of a pure-Neumann
    subdomain)."""
    ev = np.asarray(ev, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    big = np.abs(ref) > 1e-8 * scale
    d = np.abs(ev - ref)
    rel = float((d / np.where(big, np.abs(ref), 1.0))[big].max()) if big.any() else 0.0
    null = float((d / scale)[~big].max()) if (~big).any() else 0.0
    return rel, null
