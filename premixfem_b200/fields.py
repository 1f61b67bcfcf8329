"""Seeded synthetic permeability fields, boundary conditions and sources.

The reference drives its solver with a periodic "cross" channel field
(src/Expe_scal.c:11-42), an anisotropic constant field (src/test.c:7-17) and
HDF5 data sets that are not distributed with it (fracture256, SPE10).  The
benchmark configurations used here replace the missing data with seeded
synthetic fields of the same shapes and value distributions:

* ``unit_cube_grf``   32^3 unit cube, k = exp(g), g a Gaussian random field
                      (sigma 2, exponential covariance, length 0.1), p = 0 on
                      x = 1, f = 1 everywhere.
* ``layered``         60 x 220 x 85 cells of 20 x 10 x 2, smooth lognormal
                      layers on top of binary sinuous channel layers
                      (contrast 1e6), a +/-1 injector/producer pair in the
                      corner columns, no-flux walls.
* ``fracture256``     256^3 unit cells, mild lognormal background, 200
                      axis-aligned 1-cell fractures (k = 1e4) and ~5 % barrier
                      inclusions (k = 1e-4); p = 1 on x = 0, p = 0 on x = 255.
* ``large_frac``      512 x 512 x 256, anisotropic GRF (sigma 3) plus 400
                      fracture planes of contrast 1e6; p = 0 on z = 0.
* ``grf_batch``       64 independent unit-cube problems with per-axis cell
                      counts U{24..80}, k = exp(GRF) with sigma U[1,3] and
                      correlation U[0.05,0.2], p = 0 on x = 1, and 4
                      right-hand sides each (unit source + 3 N(0,1) fields).
* ``cross``           the reference's own cross field (src/Expe_scal.c:11-42).
* ``aniso_const``     the reference's test.c field k = (2, 1, 0.5).

Arrays are float64 with shape (P, N, M) = (z, y, x): x is the fastest index,
matching the DMDA natural ordering of the reference (cell id
``(ez*N + ey)*M + ex``).

A problem is a dict with keys ``mesh`` (M, N, P), ``dom`` (L, W, H),
``kappa`` (tuple of three (P,N,M) arrays, one per direction, possibly the same
array three times), ``source`` (P,N,M) cell-integrated source, ``dirichlet``
(dict face -> value, faces 'x-','x+','y-','y+','z-','z+'), ``zero_mean``.
"""
from __future__ import annotations

import numpy as np

FACES = ("x-", "x+", "y-", "y+", "z-", "z+")


def _grf_periodic(shape, spacing, sigma, corr, rng, embed=1):
    """Gaussian random field with exponential covariance sigma^2 exp(-r/corr).

    Circulant embedding on a periodic grid ``embed`` times the domain in each
    axis: the covariance is sampled on the torus, its FFT gives the circulant
    eigenvalues (negative ones clipped), and white noise is coloured by their
    square root.  ``corr`` may be a scalar or a per-axis (z, y, x) tuple for an
    anisotropic field.  Returns an array of ``shape`` with unit-variance
    scaling to ``sigma``.
    """
    shape = tuple(int(s) for s in shape)
    ext = tuple(max(2, s * embed) for s in shape)
    corr = np.broadcast_to(np.asarray(corr, dtype=np.float64), (3,))
    spacing = np.broadcast_to(np.asarray(spacing, dtype=np.float64), (3,))
    axes = []
    for a in range(3):
        n = ext[a]
        d = np.minimum(np.arange(n), n - np.arange(n)) * spacing[a] / corr[a]
        axes.append(d)
    r = np.sqrt(axes[0][:, None, None] ** 2 + axes[1][None, :, None] ** 2 + axes[2][None, None, :] ** 2)
    cov = np.exp(-r)
    lam = np.fft.rfftn(cov).real
    np.maximum(lam, 0.0, out=lam)
    w = rng.standard_normal(ext)
    f = np.fft.irfftn(np.fft.rfftn(w) * np.sqrt(lam), s=ext, axes=(0, 1, 2))
    f = f[: shape[0], : shape[1], : shape[2]]
    std = f.std()
    if std > 0:
        f = (f - f.mean()) / std
    return sigma * f


def _problem(mesh, dom, kappa, source, dirichlet=None, zero_mean=False, name=""):
    return {
        "name": name,
        "mesh": tuple(int(v) for v in mesh),
        "dom": tuple(float(v) for v in dom),
        "kappa": kappa,
        "source": source,
        "dirichlet": dict(dirichlet or {}),
        "zero_mean": bool(zero_mean),
    }


def aniso_const(M=8, N=8, P=8):
    """Constant anisotropic k = (2, 1, 0.5) with the reference's well source.

    Follows src/test.c:7-38 (create_Laplace_kappa, create_well_source_XxY_rhs).
    Pure Neumann; the source sums to zero.
    """
    shape = (P, N, M)
    kx = np.full(shape, 2.0)
    ky = np.full(shape, 1.0)
    kz = np.full(shape, 0.5)
    return _problem((M, N, P), (1.0, 1.0, 1.0), (kx, ky, kz), well_source(M, N, P, (1.0, 1.0, 1.0)),
                    zero_mean=True, name="aniso_const")


def well_source(M, N, P, dom):
    """Zero-sum well pattern of src/Expe_scal.c:44-64 (also src/test.c:19-38).

    +1e3*|K| in the four corner columns, -1e3*|K| in the four centre columns.
    """
    meas = (dom[0] / M) * (dom[1] / N) * (dom[2] / P)
    s = np.zeros((P, N, M))
    for ex in (0, M - 1):
        for ey in (0, N - 1):
            s[:, ey, ex] = 1.0e3 * meas
    cx = (M // 2 - 1, M // 2)
    cy = (N // 2 - 1, N // 2)
    for ex in cx:
        for ey in cy:
            if (ex == 0 or ex == M - 1) and (ey == 0 or ey == N - 1):
                continue
            s[:, ey, ex] = -1.0e3 * meas
    return s


def cross(size=16, cr=0):
    """The reference's periodic cross channel field (src/Expe_scal.c:11-42).

    Cells whose position modulo 8 lies in [3, 5) in two of the three axes get
    k = 10^cr, all others k = 1.  Same well source as the reference driver.
    """
    M = N = P = size
    e = np.arange(size) % 8
    inb = (e >= 3) & (e < 5)
    z = inb[:, None, None]
    y = inb[None, :, None]
    x = inb[None, None, :]
    ch = (x & y) | (x & z) | (y & z)
    k = np.where(ch, 10.0 ** cr, 1.0)
    return _problem((M, N, P), (1.0, 1.0, 1.0), (k, k, k), well_source(M, N, P, (1.0, 1.0, 1.0)),
                    zero_mean=True, name=f"cross{size}_cr{cr}")


def unit_cube_grf(n=32, seed=1, sigma=2.0, corr=0.1):
    """Unit-cube GRF problem: k = exp(g), p = 0 on x = 1, unit source."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    g = _grf_periodic((n, n, n), h, sigma, corr, rng, embed=2)
    k = np.exp(g)
    src = np.full((n, n, n), h * h * h)
    return _problem((n, n, n), (1.0, 1.0, 1.0), (k, k, k), src, {"x+": 0.0}, name=f"unit_cube_grf{n}")


def _sinuous_channels(rng, nx, ny, n_channels, wmin=3, wmax=6):
    """Binary map of sinuous channels running along y with random centre-lines."""
    mask = np.zeros((ny, nx), dtype=bool)
    yy = np.arange(ny)
    xs = np.arange(nx)
    for _ in range(n_channels):
        x0 = rng.uniform(0, nx)
        amp = rng.uniform(2.0, 10.0)
        wl = rng.uniform(30.0, 120.0)
        ph = rng.uniform(0, 2 * np.pi)
        w = rng.integers(wmin, wmax + 1)
        c = x0 + amp * np.sin(2 * np.pi * yy / wl + ph)
        mask |= np.abs(xs[None, :] - c[:, None]) < (w / 2.0)
    return mask


def layered(seed=2, M=60, N=220, P=85, smooth_layers=35, contrast=1.0e6):
    """Layered high-contrast stand-in for the SPE10-shaped benchmark.

    Layers 0..smooth_layers-1 hold a 2-D lognormal GRF (sigma 1.5, correlation
    8 cells); the remaining layers hold binary sinuous channels (width 3-6,
    contrast ``contrast``) over a low background.  Cells are 20 x 10 x 2.
    Injector (+1) in the column (0, 0), producer (-1) in (M-1, N-1), spread
    over the column; no-flux walls, so the operator is singular and the
    problem carries a zero-mean constraint.
    """
    rng = np.random.default_rng(seed)
    dom = (20.0 * M, 10.0 * N, 2.0 * P)
    k = np.empty((P, N, M))
    for z in range(P):
        if z < smooth_layers:
            g = _grf_periodic((1, N, M), 1.0, 1.5, (1.0, 8.0, 8.0), rng, embed=2)[0]
            k[z] = np.exp(g)
        else:
            ch = _sinuous_channels(rng, M, N, n_channels=int(rng.integers(3, 7)))
            k[z] = np.where(ch, np.sqrt(contrast), 1.0 / np.sqrt(contrast))
    src = np.zeros((P, N, M))
    src[:, 0, 0] = 1.0 / P
    src[:, N - 1, M - 1] = -1.0 / P
    return _problem((M, N, P), dom, (k, k, k), src, zero_mean=True, name="layered")


def _add_fractures(rng, k, n_frac, lo, hi, value):
    P, N, M = k.shape
    dims = (M, N, P)
    for _ in range(n_frac):
        normal = int(rng.integers(0, 3))
        a, b = [d for d in range(3) if d != normal]
        la = int(rng.integers(lo, hi + 1))
        lb = int(rng.integers(lo, hi + 1))
        la = min(la, dims[a])
        lb = min(lb, dims[b])
        sa = int(rng.integers(0, dims[a] - la + 1))
        sb = int(rng.integers(0, dims[b] - lb + 1))
        pos = int(rng.integers(0, dims[normal]))
        sl = [slice(None)] * 3
        # array axes are (z, y, x) = (2, 1, 0) in mesh order
        sl[2 - normal] = slice(pos, pos + 1)
        sl[2 - a] = slice(sa, sa + la)
        sl[2 - b] = slice(sb, sb + lb)
        k[tuple(sl)] = value


def _add_barriers(rng, k, frac_cells, value, smin=2, smax=6):
    P, N, M = k.shape
    target = frac_cells * k.size
    mark = np.zeros(k.shape, dtype=bool)
    count = 0
    while count < target:
        s = rng.integers(smin, smax + 1, size=3)
        z0 = int(rng.integers(0, max(1, P - s[0])))
        y0 = int(rng.integers(0, max(1, N - s[1])))
        x0 = int(rng.integers(0, max(1, M - s[2])))
        blk = mark[z0:z0 + s[0], y0:y0 + s[1], x0:x0 + s[2]]
        count += int(blk.size - blk.sum())
        blk[...] = True
    k[mark] = value


def fracture256(n=256, seed=4, n_frac=200, frac_lo=32, frac_hi=160, barrier=0.05):
    """Fracture-network stand-in for the missing fracture256 data set.

    Unit-spaced n^3 grid; background exp(0.5 * GRF) with an 8-cell correlation
    length, ``n_frac`` axis-aligned 1-cell-thick fractures of in-plane extent
    U{frac_lo..frac_hi} with k = 1e4, then box-shaped barrier inclusions with
    k = 1e-4 until ``barrier`` of the cells are covered.  p = 1 on x = 0,
    p = 0 on x = n-1, no-flux elsewhere, no volume source.
    """
    rng = np.random.default_rng(seed)
    g = _grf_periodic((n, n, n), 1.0, 0.5, 8.0, rng, embed=1)
    k = np.exp(g)
    scale = n / 256.0
    _add_fractures(rng, k, n_frac, max(2, int(frac_lo * scale)), max(2, int(frac_hi * scale)), 1.0e4)
    _add_barriers(rng, k, barrier, 1.0e-4)
    src = np.zeros((n, n, n))
    return _problem((n, n, n), (float(n), float(n), float(n)), (k, k, k), src, {"x-": 1.0, "x+": 0.0},
                    name=f"fracture{n}")


def large_frac(M=512, N=512, P=256, seed=5, n_frac=400, frac_lo=32, frac_hi=256):
    """Large anisotropic GRF + fracture planes; p = 0 on z = 0, unit source.

    Fracture planes have in-plane extent U{frac_lo..frac_hi} (clipped to the
    grid) and k = 1e6 times the background scale."""
    rng = np.random.default_rng(seed)
    g = _grf_periodic((P, N, M), (1.0 / P, 1.0 / N, 1.0 / M), 3.0, (0.02, 0.1, 0.1), rng, embed=1)
    k = np.exp(g)
    _add_fractures(rng, k, n_frac, frac_lo, frac_hi, 1.0e6)
    src = np.full((P, N, M), 1.0 / (M * N * P))
    return _problem((M, N, P), (1.0, 1.0, 1.0), (k, k, k), src, {"z-": 0.0}, name="large_frac")


def random_box(mesh, seed=0, sigma=1.0, corr=0.2, dirichlet=None, source="unit"):
    """Small seeded GRF problem on an arbitrary box, used for parity sweeps."""
    M, N, P = mesh
    rng = np.random.default_rng(seed)
    g = _grf_periodic((P, N, M), (1.0 / P, 1.0 / N, 1.0 / M), sigma, corr, rng, embed=2)
    k = np.exp(g)
    meas = 1.0 / (M * N * P)
    if source == "unit":
        src = np.full((P, N, M), meas)
    else:
        src = rng.standard_normal((P, N, M)) * meas
    if dirichlet is None:
        dirichlet = {"x-": 0.0}
    return _problem((M, N, P), (1.0, 1.0, 1.0), (k, k, k), src, dirichlet, zero_mean=not dirichlet,
                    name=f"random{M}x{N}x{P}")


def grf_batch(count=64, seed=3, lo=24, hi=80, n_rhs=4):
    """The batching workload: ``count`` independent problems on the unit cube.

    Per problem: per-axis cell counts U{lo..hi}; k = exp(g), g a GRF with
    sigma U[1,3] and isotropic exponential correlation length U[0.05,0.2];
    p = 0 on x = 1, no-flux elsewhere.  Right-hand sides: the unit source
    f = 1 and ``n_rhs - 1`` fields of N(0,1) values, all cell-integrated.
    Returns a list of (problem, [source arrays]); ``problem["source"]`` is the
    unit source.
    """
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        M, N, P = (int(v) for v in rng.integers(lo, hi + 1, size=3))
        sigma = float(rng.uniform(1.0, 3.0))
        corr = float(rng.uniform(0.05, 0.2))
        g = _grf_periodic((P, N, M), (1.0 / P, 1.0 / N, 1.0 / M), sigma, corr, rng, embed=2)
        k = np.exp(g)
        meas = 1.0 / (M * N * P)
        sources = [np.full((P, N, M), meas)]
        for _ in range(n_rhs - 1):
            sources.append(rng.standard_normal((P, N, M)) * meas)
        prob = _problem((M, N, P), (1.0, 1.0, 1.0), (k, k, k), sources[0], {"x+": 0.0},
                        name=f"grf_batch{M}x{N}x{P}")
        out.append((prob, sources))
    return out


def tiles(mesh, tile=8):
    """Subdomains per axis for tiles of about ``tile`` cells (near-equal split,
    so boundary-adjacent sizes are ragged): ceil(n / tile), at least 2."""
    return tuple(max(2, -(-int(n) // tile)) for n in mesh)
