"""Seeded synthetic CRS problems for the PARCEL-legacy Krylov path.

Every generator returns a :class:`CRS` in the reference's layout: 1-based row pointer
(``crsRow_ptr(1) = 1``), 1-based global column ids sorted within each row, ``float64``
values and ``int32`` indices (src/define.f90:133-164).  Random inputs come from
``numpy.random.default_rng(seed)`` (PCG64), so a seed fixes every array bit for bit.

The stencil generators emit a row's entries in increasing column order
(bottom, south, west, centre, east, north, top), which is also the order the reference's
own generator uses (src/example/problem.f90:448-618).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class CRS:
    n: int
    rowptr: np.ndarray  # int32, n+1, 1-based
    col: np.ndarray     # int32, nnz, 1-based
    val: np.ndarray     # float64, nnz
    istart: int = 1

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col - 1, self.rowptr - 1), shape=(self.n, self.n))


def _assemble(n: int, cols: list, vals: list, masks: list) -> CRS:
    """Builds CRS from per-offset column/value/mask arrays given in column order."""
    C = np.stack(cols, axis=1)
    V = np.stack(vals, axis=1)
    M = np.stack(masks, axis=1)
    counts = M.sum(axis=1, dtype=np.int64)
    rowptr = np.empty(n + 1, dtype=np.int64)
    rowptr[0] = 1
    np.cumsum(counts, out=rowptr[1:])
    rowptr[1:] += 1
    col = C[M].astype(np.int32) + 1
    val = V[M].astype(np.float64)
    return CRS(n=n, rowptr=rowptr.astype(np.int32), col=col, val=val)


def _grid3(nx: int, ny: int, nz: int):
    i = np.arange(nx * ny * nz, dtype=np.int64)
    ix = i % nx
    iy = (i // nx) % ny
    iz = i // (nx * ny)
    return i, ix, iy, iz


def poisson3d_reference(gnx: int, gny: int, gnz: int):
    """The reference's own golden problem on one process.

    Matrix: make_poisson3D_CRS (src/example/problem.f90:448-618) with dx=dy=dz=1:
    diagonal -6, off-diagonals +1, Dirichlet rows truncated (negative definite).
    RHS and exact solution: make_poisson3D_right_vector (problem.f90:772-875),
    x* = h^6 (ix iy iz)^2 with h = 1/(g+1) per axis.
    Returns (A, b, x_exact).
    """
    n = gnx * gny * gnz
    i, ix, iy, iz = _grid3(gnx, gny, gnz)
    sxy = gnx * gny
    one = np.ones(n)
    cols = [i - sxy, i - gnx, i - 1, i, i + 1, i + gnx, i + sxy]
    vals = [one, one, one, -6.0 * one, one, one, one]
    masks = [iz > 0, iy > 0, ix > 0, np.ones(n, bool), ix < gnx - 1, iy < gny - 1, iz < gnz - 1]
    A = _assemble(n, cols, vals, masks)

    hx, hy, hz = 1.0 / (gnx + 1), 1.0 / (gny + 1), 1.0 / (gnz + 1)
    X = (ix + 1).astype(np.float64) ** 2
    Y = (iy + 1).astype(np.float64) ** 2
    Z = (iz + 1).astype(np.float64) ** 2
    z = 2.0 * (hx ** 2) * (hy ** 2) * (hz ** 2)
    b = z * (X * Y + Y * Z + Z * X)
    m = ix == gnx - 1
    b[m] = b[m] - (hy * (iy[m] + 1)) ** 2 * (hz * (iz[m] + 1)) ** 2
    m = iy == gny - 1
    b[m] = b[m] - (hx * (ix[m] + 1)) ** 2 * (hz * (iz[m] + 1)) ** 2
    m = iz == gnz - 1
    b[m] = b[m] - (hx * (ix[m] + 1)) ** 2 * (hy * (iy[m] + 1)) ** 2
    zx = (hx ** 2) * (hy ** 2) * (hz ** 2)
    x_exact = zx * (X * Y * Z)
    return A, b, x_exact


def poisson2d_5pt(nx: int, ny: int) -> CRS:
    """2D 5-point Poisson, 4 on the diagonal, -1 off it, Dirichlet (rows truncated)."""
    n = nx * ny
    i = np.arange(n, dtype=np.int64)
    ix, iy = i % nx, i // nx
    one = np.ones(n)
    cols = [i - nx, i - 1, i, i + 1, i + nx]
    vals = [-one, -one, 4.0 * one, -one, -one]
    masks = [iy > 0, ix > 0, np.ones(n, bool), ix < nx - 1, iy < ny - 1]
    return _assemble(n, cols, vals, masks)


def convdiff3d_upwind(N: int, peclet: float = 10.0, v=(1.0, 0.5, 0.25)) -> CRS:
    """-Laplace(u) + Pe v.grad(u) on the unit cube, N^3 interior cells, h = 1/(N+1),
    first-order upwind differences, Dirichlet boundary, scaled by h^2.

    Row i: diagonal 6 + Pe h (|vx|+|vy|+|vz|); the upwind neighbour along each axis gets
    -1 - Pe h |v|, the downwind one -1.
    """
    n = N ** 3
    h = 1.0 / (N + 1)
    i, ix, iy, iz = _grid3(N, N, N)
    c = [peclet * h * abs(vv) for vv in v]
    one = np.ones(n)
    # upwind side is "minus" for positive velocity components
    lo = [-1.0 - (c[k] if v[k] > 0 else 0.0) for k in range(3)]
    hi = [-1.0 - (c[k] if v[k] < 0 else 0.0) for k in range(3)]
    diag = 6.0 + sum(c)
    S = N * N
    cols = [i - S, i - N, i - 1, i, i + 1, i + N, i + S]
    vals = [lo[2] * one, lo[1] * one, lo[0] * one, diag * one, hi[0] * one, hi[1] * one, hi[2] * one]
    masks = [iz > 0, iy > 0, ix > 0, np.ones(n, bool), ix < N - 1, iy < N - 1, iz < N - 1]
    return _assemble(n, cols, vals, masks)


def aniso3d(N: int, k=(1.0, 1.0e-2, 1.0e-4)) -> CRS:
    """Anisotropic 7-point diffusion, coefficients (kx, ky, kz), unit spacing, Dirichlet.
    Diagonal 2(kx+ky+kz), neighbours -k along their axis."""
    n = N ** 3
    i, ix, iy, iz = _grid3(N, N, N)
    one = np.ones(n)
    S = N * N
    kx, ky, kz = k
    cols = [i - S, i - N, i - 1, i, i + 1, i + N, i + S]
    vals = [-kz * one, -ky * one, -kx * one, 2.0 * (kx + ky + kz) * one, -kx * one, -ky * one, -kz * one]
    masks = [iz > 0, iy > 0, ix > 0, np.ones(n, bool), ix < N - 1, iy < N - 1, iz < N - 1]
    return _assemble(n, cols, vals, masks)


def banded_random(n: int, bandwidth: int = 64, nnz_row: int = 9, seed: int = 4,
                  diag_factor: float = 1.2) -> CRS:
    """Random nonsymmetric banded matrix: the diagonal plus nnz_row-1 distinct
    off-diagonal offsets per row drawn uniformly from the valid offsets in
    [-bandwidth, bandwidth] minus {0}; off-diagonal values U[-1,1); the diagonal is
    diag_factor times the row's absolute off-diagonal sum."""
    rng = np.random.default_rng(seed)
    k = nnz_row - 1
    i = np.arange(n, dtype=np.int64)
    lo = np.maximum(-bandwidth, -i)             # most negative valid offset
    hi = np.minimum(bandwidth, n - 1 - i)       # most positive valid offset
    ncand = (hi - lo)                           # candidates excluding 0
    if np.any(ncand < k):
        raise ValueError("matrix too small for the requested band")
    # Floyd's sampling of k distinct indices in [0, ncand) per row
    S = np.empty((n, k), dtype=np.int64)
    for j in range(k):
        top = ncand - k + j                     # sample t in [0, top]
        t = np.floor(rng.random(n) * (top + 1)).astype(np.int64)
        dup = (S[:, :j] == t[:, None]).any(axis=1) if j else np.zeros(n, bool)
        S[:, j] = np.where(dup, top, t)
    off = lo[:, None] + S
    off = np.where(off >= 0, off + 1, off)      # skip the diagonal
    vals = rng.random((n, k)) * 2.0 - 1.0
    cols = i[:, None] + off
    allc = np.concatenate([cols, i[:, None]], axis=1)
    allv = np.concatenate([vals, np.zeros((n, 1))], axis=1)
    order = np.argsort(allc, axis=1, kind="stable")
    allc = np.take_along_axis(allc, order, axis=1)
    allv = np.take_along_axis(allv, order, axis=1)
    dmask = allc == i[:, None]
    rowsum = np.abs(allv).sum(axis=1)
    allv[dmask] = diag_factor * rowsum
    rowptr = (np.arange(n + 1, dtype=np.int64) * nnz_row + 1).astype(np.int32)
    return CRS(n=n, rowptr=rowptr, col=(allc.reshape(-1) + 1).astype(np.int32),
               val=allv.reshape(-1).astype(np.float64))


def gaussian_random_field(N: int, corr_len: float = 8.0, variance: float = 2.0,
                          seed: int = 5) -> np.ndarray:
    """Stationary Gaussian random field on an N^3 periodic grid: white noise filtered
    with a Gaussian kernel of correlation length corr_len cells (FFT), rescaled to the
    requested variance and zero mean.  Returns float64 (N, N, N) indexed [z, y, x]."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((N, N, N))
    f = np.fft.fftfreq(N)
    kz, ky, kx = np.meshgrid(f, f, np.fft.rfftfreq(N), indexing="ij")
    k2 = kx ** 2 + ky ** 2 + kz ** 2
    filt = np.exp(-2.0 * (np.pi * corr_len) ** 2 * k2 / 2.0)
    g = np.fft.irfftn(np.fft.rfftn(w) * filt, s=(N, N, N), axes=(0, 1, 2))
    g -= g.mean()
    g *= np.sqrt(variance) / g.std()
    return g


def vardiff3d(N: int, coeff: np.ndarray) -> CRS:
    """Variable-coefficient 7-point diffusion with harmonic-mean face coefficients,
    following make_poisson3D_adv_CRS (src/example/problem.f90:620-770) with
    dx = dy = dz = 1/N: the off-diagonal towards a neighbour is
    -h / (0.5 (1/k_c + 1/k_nb)) and the diagonal is minus their sum, boundary faces
    included (the ghost cell takes the boundary cell's coefficient); off-diagonals
    pointing outside the grid are dropped.  The matrix is symmetric positive definite.
    coeff is indexed [z, y, x]."""
    n = N ** 3
    h = 1.0 / N
    kc = coeff.reshape(-1)
    i, ix, iy, iz = _grid3(N, N, N)
    kp = np.pad(coeff, 1, mode="edge")
    def face(dz, dy, dx):
        nb = kp[1 + dz:1 + dz + N, 1 + dy:1 + dy + N, 1 + dx:1 + dx + N].reshape(-1)
        return -h / (0.5 * (1.0 / kc + 1.0 / nb))
    cb, cs, cw = face(-1, 0, 0), face(0, -1, 0), face(0, 0, -1)
    ct, cn, ce = face(1, 0, 0), face(0, 1, 0), face(0, 0, 1)
    cc = -(cw + ce + cs + cn + cb + ct)
    S = N * N
    cols = [i - S, i - N, i - 1, i, i + 1, i + N, i + S]
    vals = [cb, cs, cw, cc, ce, cn, ct]
    masks = [iz > 0, iy > 0, ix > 0, np.ones(n, bool), ix < N - 1, iy < N - 1, iz < N - 1]
    return _assemble(n, cols, vals, masks)


def rhs_uniform(n: int, seed: int) -> np.ndarray:
    """b ~ U[-1, 1)."""
    return np.random.default_rng(seed).random(n) * 2.0 - 1.0


def rhs_normal(n: int, seed: int, nrhs: int = 1) -> np.ndarray:
    """b ~ N(0, 1); shape (n,) or (nrhs, n)."""
    r = np.random.default_rng(seed).standard_normal((nrhs, n) if nrhs > 1 else n)
    return r
