"""The two-level stage's coarse-grid kernels on the GPU against oracle/coarse.py, through the
C-ABI: the Galerkin operator (FP64, summed in a different order: 1e-12 of the largest
entry), the transfers (FP32 arithmetic: 1e-6 relative) and the one-cluster coarse PCG
(FP32 vectors: 1e-4 relative after a few iterations, 2e-3 after twenty, against the
float64 restatement of the same recurrence)."""
import numpy as np
import pytest

import coarse
from parcel_b import api, problems

pytestmark = pytest.mark.gpu


def _vardiff(N, seed):
    g = problems.gaussian_random_field(N, corr_len=N / 8.0, variance=2.0, seed=seed)
    return problems.vardiff3d(N, np.exp(g))


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("case", ["poisson_16x12x8_c4", "convdiff16_c4", "vardiff16_c8", "vardiff24_c2"])
def test_galerkin_matches_oracle(case):
    if case == "poisson_16x12x8_c4":
        (nx, ny, nz), c = (16, 12, 8), 4
        A, _, _ = problems.poisson3d_reference(nx, ny, nz)
    elif case == "convdiff16_c4":
        (nx, ny, nz), c = (16, 16, 16), 4
        A = problems.convdiff3d_upwind(16)
    elif case == "vardiff16_c8":
        (nx, ny, nz), c = (16, 16, 16), 8
        A = _vardiff(16, 3)
    else:
        (nx, ny, nz), c = (24, 24, 24), 2
        A = _vardiff(24, 4)
    h = api.Learned(nx, ny, nz, c)
    ac = h.galerkin(A)
    ao = coarse.galerkin27(A, nx, ny, nz, c)
    assert np.max(np.abs(ac - ao)) <= 1e-12 * np.max(np.abs(ao))


def test_transfers_match_oracle():
    nx, ny, nz, c = 32, 16, 24, 4
    h = api.Learned(nx, ny, nz, c)
    P = coarse.prolongation(nx, ny, nz, c)
    rng = np.random.default_rng(7)
    v = rng.standard_normal(nx * ny * nz)
    y = rng.standard_normal(P.shape[1])
    assert _rel(h.restrict(v), P.T @ v) < 1e-6
    assert _rel(h.prolong(y), P @ y) < 1e-6


@pytest.mark.parametrize("N,c", [(32, 4), (128, 4)])
def test_coarse_pcg_matches_oracle(N, c):
    """32^3 / 4: one coarse plane per CTA of the cluster; 128^3 / 4: a 32^3 coarse grid, four
    coarse cells per thread."""
    A = _vardiff(N, 6)
    h = api.Learned(N, N, N, c)
    ao = coarse.galerkin27(A, N, N, N, c)
    G = N // c
    rng = np.random.default_rng(8)
    rc = rng.standard_normal(G ** 3).astype(np.float32)
    for steps, tol in ((1, 1e-4), (5, 1e-4), (20, 2e-3)):
        y = h.coarse_solve(A, rc, steps)
        yo = coarse.pcg(ao, (G, G, G), rc.astype(np.float64), steps)
        assert _rel(y, yo) < tol, (steps, _rel(y, yo))
    # a starting guess is rescaled by the energy-optimal gamma, then iterated
    g0 = (coarse.pcg(ao, (G, G, G), rc.astype(np.float64), 3) * 7.0).astype(np.float32)
    for steps in (0, 4):
        y = h.coarse_solve(A, rc, steps, g0=g0)
        yo = coarse.pcg(ao, (G, G, G), rc.astype(np.float64), steps, g0=g0.astype(np.float64))
        assert _rel(y, yo) < 1e-4, (steps, _rel(y, yo))
