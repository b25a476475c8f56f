"""Self-checks of the coarse-grid restatement (oracle/coarse.py) that the GPU stage is tested
against.  The two-level stage has no counterpart in the reference, so these properties pin
the oracle: P reproduces fields linear in the cell centres, the restriction is P's
transpose, the Galerkin operator of a symmetric matrix is symmetric and has the row sums of
P^T A P, the 27-tap product equals the sparse product, and enough coarse PCG iterations
solve the coarse system."""
import numpy as np
import scipy.sparse.linalg as spla

import coarse
from parcel_b import problems


def _vardiff(nx, ny, nz, seed):
    assert nx == ny == nz
    g = problems.gaussian_random_field(nx, corr_len=nx / 8.0, variance=2.0, seed=seed)
    return problems.vardiff3d(nx, np.exp(g))


def test_prolongation_reproduces_linear_fields_inside_and_sums_to_one():
    nx, ny, nz, c = 16, 8, 12, 4
    P = coarse.prolongation(nx, ny, nz, c)
    assert np.allclose(P @ np.ones(P.shape[1]), 1.0)
    gx, gy, gz = nx // c, ny // c, nz // c
    I = np.arange(gx * gy * gz)
    cx, cy, cz = I % gx, (I // gx) % gy, I // (gx * gy)
    lin = 2.0 * cx - 3.0 * cy + 0.5 * cz
    f = (P @ lin).reshape(nz, ny, nx)
    x = (np.arange(nx) + 0.5) / c - 0.5
    y = (np.arange(ny) + 0.5) / c - 0.5
    z = (np.arange(nz) + 0.5) / c - 0.5
    # away from the clamped boundary layer the interpolant is the linear field itself
    sl = (slice(c // 2, nz - c // 2), slice(c // 2, ny - c // 2), slice(c // 2, nx - c // 2))
    want = 2.0 * x[None, None, :] - 3.0 * y[None, :, None] + 0.5 * z[:, None, None]
    assert np.allclose(f[sl], want[sl])


def test_galerkin27_keeps_symmetry_and_matches_the_sparse_product():
    N, c = 16, 4
    A = _vardiff(N, N, N, 3)
    ac = coarse.galerkin27(A, N, N, N, c)
    G = N // c
    # symmetric: tap t of cell I equals tap 26 - t of the neighbour I + d
    for t in range(27):
        dx, dy, dz = t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1
        for I in range(G ** 3):
            x, y, z = I % G, (I // G) % G, I // (G * G)
            jx, jy, jz = x + dx, y + dy, z + dz
            if 0 <= jx < G and 0 <= jy < G and 0 <= jz < G:
                J = (jz * G + jy) * G + jx
                assert abs(ac[t, I] - ac[26 - t, J]) <= 1e-12 * abs(ac[13, I])
            else:
                assert ac[t, I] == 0.0
    # the 27-tap product equals the truncated sparse product
    P = coarse.prolongation(N, N, N, c)
    Ac = (P.T @ A.to_scipy() @ P).toarray()
    v = np.random.default_rng(0).standard_normal(G ** 3)
    full = Ac @ v
    taps = coarse.apply27(ac, G, G, G, v)
    # the dropped couplings (two coarse cells apart) are small next to the kept ones
    assert np.linalg.norm(taps - full) < 0.05 * np.linalg.norm(full)


def test_pcg_solves_the_coarse_system_and_uses_the_guess():
    N, c = 32, 4
    A = _vardiff(N, N, N, 5)
    ac = coarse.galerkin27(A, N, N, N, c)
    G = N // c
    rc = np.random.default_rng(1).standard_normal(G ** 3)
    y = coarse.pcg(ac, (G, G, G), rc, 400)
    assert np.linalg.norm(coarse.apply27(ac, G, G, G, y) - rc) < 1e-8 * np.linalg.norm(rc)
    # the exact solution as the guess: gamma = 1 and nothing left to do
    y0 = coarse.pcg(ac, (G, G, G), rc, 0, g0=y)
    assert np.allclose(y0, y, rtol=1e-7, atol=1e-12 * np.abs(y).max())


def test_restriction_is_the_transpose_of_prolongation():
    nx, ny, nz, c = 8, 12, 16, 4
    P = coarse.prolongation(nx, ny, nz, c)
    rng = np.random.default_rng(2)
    v, w = rng.standard_normal(P.shape[0]), rng.standard_normal(P.shape[1])
    assert np.isclose((P.T @ v) @ w, v @ (P @ w))
