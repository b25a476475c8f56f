"""Headroom of the coarse-grid stage (CPU, numpy/scipy): what the stage formulation of the
learned FGMRES preconditioner gains when its coarse problem is solved exactly.

The stage after the block-Jacobi ILU(0) z1 = M r is t = r - A z1, c = P A_c^-1 R t,
z = z1 + alpha c with alpha = <t, A c> / <A c, A c>.  The learned stage replaces A_c^-1 R
by the network on the coarse grid; here A_c = P^T A P (Galerkin, P the cell-centred
trilinear prolongation of oracle/cnn.py) is factorised exactly, which bounds what any
one-level coarse stage at that coarsening can do.  On the 64^3 variable-coefficient
problem of the learned benchmark (k = exp(GRF), correlation 8 cells, variance 2) it cuts
the FGMRES(40) iterations about 2.7x at c = 8 and 5x at c = 4, and 2 / 6 steps of
Jacobi-preconditioned CG on the coarse operator in place of the exact solve already give
3.2x / 4.6x at c = 4; at 128^3 (too slow for this suite) the same study gives 8.9x and
16.5x for the exact solve and 4.3x / 7.7x / 8.8x for 2 / 4 / 8 coarse PCG steps at c = 8,
against about 1.7x for the trained network at 256^3.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle
from parcel_b import problems


def _interp1d(N, c):
    """1-D cell-centred linear interpolation (N fine x N/c coarse), clamped at the ends;
    the Kronecker cube of it is oracle/cnn.py's prolong()."""
    G = N // c
    i = np.arange(N)
    xi = (i + 0.5) / c - 0.5
    i0 = np.floor(xi).astype(int)
    w = xi - i0
    lo, hi = np.clip(i0, 0, G - 1), np.clip(i0 + 1, 0, G - 1)
    return sp.coo_matrix((np.r_[1 - w, w], (np.r_[i, i], np.r_[lo, hi])), shape=(N, G)).tocsr()


def _fgmres(A, b, prec, m=40, tol=1e-10, maxit=2000):
    n = len(b)
    x = np.zeros(n)
    bn = np.linalg.norm(b)
    it = 0
    while it < maxit:
        r = b - A @ x
        beta = np.linalg.norm(r)
        if beta / bn < tol:
            break
        V, Z, H = np.zeros((m + 1, n)), np.zeros((m, n)), np.zeros((m + 1, m))
        V[0] = r / beta
        g = np.zeros(m + 1)
        g[0] = beta
        cs, sn = np.zeros(m), np.zeros(m)
        for j in range(m):
            Z[j] = prec(V[j])
            w = A @ Z[j]
            for i in range(j + 1):
                H[i, j] = w @ V[i]
                w -= H[i, j] * V[i]
            H[j + 1, j] = np.linalg.norm(w)
            V[j + 1] = w / H[j + 1, j]
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            d = np.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = H[j, j] / d, H[j + 1, j] / d
            H[j, j], H[j + 1, j] = d, 0.0
            g[j + 1], g[j] = -sn[j] * g[j], cs[j] * g[j]
            it += 1
            if abs(g[j + 1]) / bn < tol or it >= maxit:
                break
        k = j + 1
        x += Z[:k].T @ np.linalg.solve(np.triu(H[:k, :k]), g[:k])
        if abs(g[k]) / bn < tol:
            break
    return x, it


def _pcg_k(Ac, rhs, k, dinv):
    """k steps of Jacobi-preconditioned CG on the coarse operator from a zero guess."""
    x = np.zeros_like(rhs)
    r = rhs.copy()
    z = dinv * r
    p = z.copy()
    rz = r @ z
    for _ in range(k):
        q = Ac @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        z = dinv * r
        rz2 = r @ z
        p = z + (rz2 / rz) * p
        rz = rz2
    return x


def test_exact_coarse_stage_headroom_64cube():
    N = 64
    g = problems.gaussian_random_field(N, corr_len=8.0, variance=2.0, seed=5)
    Acrs = problems.vardiff3d(N, np.exp(g))
    A = Acrs.to_scipy()
    b = problems.rhs_normal(A.shape[0], 1)
    M = oracle.Precon(oracle.Matrix(Acrs), ipreflag=2, ILU_method=0, precon_thblock=64)
    x, it0 = _fgmres(A, b, M)
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 2e-10
    gains = {}
    for c in (8, 4):
        P1 = _interp1d(N, c)
        P = sp.kron(sp.kron(P1, P1), P1).tocsr()
        lu = spla.splu((P.T @ A @ P).tocsc())

        def stage(v, P=P, lu=lu):
            z1 = M(v)
            t = v - A @ z1
            cc = P @ lu.solve(P.T @ t)
            q = A @ cc
            return z1 + (t @ q) / (q @ q) * cc

        x, it = _fgmres(A, b, stage)
        assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 2e-10
        gains[c] = it0 / it
    assert gains[8] > 2.4 and gains[4] > 4.5, (it0, gains)
    # a few Jacobi-PCG steps on the coarse operator (reach k coarse cells) recover most of it
    Ac = (P.T @ A @ P).tocsr()
    dinv = 1.0 / Ac.diagonal()
    for k, want in ((2, 2.8), (6, 4.2)):
        def stage_k(v, k=k):
            z1 = M(v)
            t = v - A @ z1
            cc = P @ _pcg_k(Ac, P.T @ t, k, dinv)
            q = A @ cc
            return z1 + (t @ q) / (q @ q) * cc

        _, it = _fgmres(A, b, stage_k)
        assert it0 / it > want, (k, it0, it)
