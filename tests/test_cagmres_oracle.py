"""The CA-GMRES oracle (oracle/cagmres.py) against GMRES(s*t) of the C oracle.

In exact arithmetic CA-GMRES(s, t) produces the iterates of GMRES(m = s*t): same Krylov
space, same least-squares problem at every basis vector.  The residual histories of the
two oracles must therefore agree to rounding level wherever the s-step basis stays well
conditioned, for every basis and QR variant of the reference.
"""
import numpy as np
import pytest

import cagmres
import oracle
from parcel_b import problems


@pytest.fixture(scope="module")
def convdiff():
    A = problems.convdiff3d_upwind(10)
    return A, problems.rhs_normal(A.n, 2)


@pytest.mark.parametrize("s,t,basis,qr,pre", [
    (4, 1, cagmres.MONOMIAL, cagmres.QR_CHOL, dict(ipreflag=1)),
    (4, 2, cagmres.MONOMIAL, cagmres.QR_CHOL2, dict(ipreflag=1)),
    (2, 4, cagmres.MONOMIAL, cagmres.QR_TSQR, dict(ipreflag=2, ILU_method=0, precon_thblock=4)),
    (4, 3, cagmres.NEWTON, cagmres.QR_CHOL2, dict(ipreflag=1)),
    (8, 4, cagmres.NEWTON, cagmres.QR_TSQR, dict(ipreflag=1)),
])
def test_cagmres_equals_gmres_st(convdiff, s, t, basis, qr, pre):
    A, b = convdiff
    xg, hg, ng, ig = oracle.solve(A, b, solver=3, GMRES_m=s * t, GMRES_GSflag=1, itrmax=800, rtolmax=1e-10, **pre)
    xc, hc, nc, ic = cagmres.pcagmres(A, b, s=s, t=t, basis=basis, qrflag=qr, itrmax=800, rtolmax=1e-10, **pre)
    assert ig == 0 and ic == 0
    assert abs(nc - ng) <= 1
    k = min(len(hg), len(hc))
    m = hg[:k] > 1e-8     # before the s-step basis' rounding floor
    assert np.max(np.abs(hc[:k][m] - hg[:k][m]) / hg[:k][m]) < 1e-6
    assert oracle.true_relres(A, b, xc) < 1e-9


def test_leja_ordering_keeps_conjugate_pairs_together():
    er = np.array([1.0, 3.0, 3.0, -2.0, 0.5])
    ei = np.array([0.0, 1.0, -1.0, 0.0, 0.0])
    wr, wi = cagmres.leja(er, ei)
    assert sorted(np.round(wr + 1j * wi, 12), key=lambda z: (z.real, z.imag)) == \
        sorted(np.round(er + 1j * ei, 12), key=lambda z: (z.real, z.imag))
    for i in range(len(wi)):
        if wi[i] > 0:
            assert wi[i + 1] == -wi[i] and wr[i + 1] == wr[i]


def test_dd_oracle_is_more_accurate_than_double():
    from fractions import Fraction
    import dd
    rng = np.random.default_rng(0)
    a, b = rng.standard_normal(200), rng.standard_normal(200)
    h, l = dd.mul(a, np.zeros(200), b, np.zeros(200))
    for i in range(20):
        exact = Fraction(a[i]) * Fraction(b[i])
        assert Fraction(h[i]) + Fraction(l[i]) == exact      # dd product of doubles is exact
