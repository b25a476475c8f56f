"""CPU restatement of the two-level preconditioner stage's coarse-grid operators.

Test infrastructure only: the GPU library (parcel-legacy_b200/csrc/pb_coarse.cu) is checked
against these functions; nothing in the product imports this module.  The stage has no
counterpart in the reference (PARCEL's preconditioners are one-level: point Jacobi,
block-Jacobi ILU / D-ILU, additive Schwarz; src/matrix.f90), so its parity is anchored on
self-checks in tests/test_coarse_oracle.py instead of reference outputs (parity unpinned
against the reference): P^T A P of a symmetric matrix is symmetric, P reproduces fields
linear in the cell centres, the restriction is P's transpose, and the coarse PCG with
enough iterations solves A_c y = rc.

Grid: natural row (z ny + y) nx + x; coarsening factor c (even) along every axis; coarse
grid (gx, gy, gz) = (nx, ny, nz) / c.  P: cell-centred trilinear interpolation clamped at
the boundary (fine cell i sits at u = (i + 1/2) / c - 1/2 in coarse units and takes
weight 1 - w from clamp(floor(u)) and w = u - floor(u) from clamp(floor(u) + 1)).
A_c = P^T A P restricted to the 27 couplings with coarse offsets in {-1, 0, 1}^3, stored
as ac[27][Vc] with tap t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def interp1d(N: int, c: int):
    """N x N/c matrix of the 1-D cell-centred linear interpolation, clamped at the ends."""
    G = N // c
    i = np.arange(N)
    num = 2 * i + 1 - c
    i0 = np.floor_divide(num, 2 * c)
    w = (num - 2 * c * i0) / (2.0 * c)
    lo, hi = np.clip(i0, 0, G - 1), np.clip(i0 + 1, 0, G - 1)
    return sp.coo_matrix((np.r_[1 - w, w], (np.r_[i, i], np.r_[lo, hi])), shape=(N, G)).tocsr()


def prolongation(nx: int, ny: int, nz: int, c: int):
    """P (n x Vc) for the natural ordering (x fastest)."""
    return sp.kron(interp1d(nz, c), sp.kron(interp1d(ny, c), interp1d(nx, c))).tocsr()


def galerkin27(A, nx: int, ny: int, nz: int, c: int) -> np.ndarray:
    """ac[27][Vc]: the couplings of P^T A P between coarse cells at most one apart per axis.
    A: scipy sparse (n x n) or an object with to_scipy()."""
    if hasattr(A, "to_scipy"):
        A = A.to_scipy()
    P = prolongation(nx, ny, nz, c)
    Ac = (P.T @ A @ P).tocoo()
    gx, gy, gz = nx // c, ny // c, nz // c
    I, J = Ac.row, Ac.col
    d = [(J % gx) - (I % gx), (J // gx) % gy - (I // gx) % gy, J // (gx * gy) - I // (gx * gy)]
    keep = (np.abs(d[0]) <= 1) & (np.abs(d[1]) <= 1) & (np.abs(d[2]) <= 1)
    t = 9 * (d[2] + 1) + 3 * (d[1] + 1) + (d[0] + 1)
    ac = np.zeros((27, gx * gy * gz))
    np.add.at(ac, (t[keep], I[keep]), Ac.data[keep])
    return ac


def apply27(ac: np.ndarray, gx: int, gy: int, gz: int, p: np.ndarray) -> np.ndarray:
    """q = A_c p from the 27-tap array."""
    P = p.reshape(gz, gy, gx)
    q = np.zeros_like(P)
    A = ac.reshape(27, gz, gy, gx)
    for t in range(27):
        dx, dy, dz = t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1
        src = np.zeros_like(P)
        zs = slice(max(0, -dz), gz - max(0, dz))
        ys = slice(max(0, -dy), gy - max(0, dy))
        xs = slice(max(0, -dx), gx - max(0, dx))
        zt = slice(max(0, dz), gz - max(0, -dz))
        yt = slice(max(0, dy), gy - max(0, -dy))
        xt = slice(max(0, dx), gx - max(0, -dx))
        src[zs, ys, xs] = P[zt, yt, xt]
        q += A[t] * src
    return q.reshape(-1)


def pcg(ac: np.ndarray, grid, rc: np.ndarray, steps: int, g0: np.ndarray | None = None) -> np.ndarray:
    """`steps` Jacobi-PCG iterations on A_c y = rc in float64: from zero, or from gamma g0
    with gamma = <rc, g0> / <g0, A_c g0>.  Same recurrence and stop rules as the GPU
    kernel (stop when <r, D^-1 r> or <p, A_c p> is exactly zero)."""
    gx, gy, gz = grid
    d = ac[13]
    dinv = np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 0.0)
    r = np.array(rc, dtype=np.float64)
    y = np.zeros_like(r)
    if g0 is not None:
        g = np.asarray(g0, np.float64)
        q = apply27(ac, gx, gy, gz, g)
        s0, s1 = float(r @ g), float(g @ q)
        gam = s0 / s1 if s1 != 0 and np.isfinite(s0 / s1) else 0.0
        y = gam * g
        r = r - gam * q
    p = dinv * r
    rz = float(r @ p)
    for _ in range(steps):
        if not abs(rz) > 0:
            break
        q = apply27(ac, gx, gy, gz, p)
        pq = float(p @ q)
        if not abs(pq) > 0:
            break
        alpha = rz / pq
        y = y + alpha * p
        r = r - alpha * q
        rz1 = float(r @ (dinv * r))
        p = dinv * r + (rz1 / rz) * p
        rz = rz1
    return y
