"""The oracle's double-double BiCGStab and GMRES(m) against its FP64 solvers (CPU).

No stored reference output covers ddKSP_pBiCG or ddKSP_pGMRES, so their restatements are
checked against the double-precision restatements of KSP_pBiCG / KSP_pGMRES (themselves
pinned through the GPU parity tests): the same algorithm in more precise arithmetic must
take the same number of iterations on a well-conditioned problem, follow the same residual
history to the accuracy of the FP64 solve, and reach the requested true residual.
"""
import numpy as np
import pytest

import oracle
from parcel_b import problems


def _system(g, seed):
    A = problems.convdiff3d_upwind(g)
    return A, problems.rhs_normal(A.n, seed)


PRECON = [dict(ipreflag=2, ILU_method=1, precon_thblock=8), dict(ipreflag=1), dict(ipreflag=0)]


@pytest.mark.parametrize("case", PRECON, ids=["dilu-8", "point-jacobi", "none"])
def test_ddbicgstab_follows_fp64_bicgstab(case):
    A, b = _system(16, 3)
    kw = dict(itrmax=300, rtolmax=1e-11, **case)
    xh, xl, h, n, ir = oracle.ddcg(A, b, solver=2, **kw)
    _, h64, n64, ir64 = oracle.solve(A, b, solver=2, **kw)
    assert ir == ir64 == 0 and abs(n - n64) <= 1
    # BiCGStab amplifies the FP64 solve's rounding as it converges, so the histories are
    # compared while the residual is above 1e-4 (later they differ by up to 1e-3 without a
    # preconditioner, because of the FP64 run)
    k = min(n, n64)
    above = h64[:k] > 1e-4
    assert np.max(np.abs(h[:k] - h64[:k])[above] / h64[:k][above]) < 1e-7
    assert oracle.true_relres(A, b, xh + xl) < 1e-10


@pytest.mark.parametrize("gs", [1, 2], ids=["mgs", "cgs"])
@pytest.mark.parametrize("case", PRECON, ids=["dilu-8", "point-jacobi", "none"])
def test_ddgmres_follows_fp64_gmres(case, gs):
    A, b = _system(16, 4)
    kw = dict(itrmax=400, rtolmax=1e-11, GMRES_m=10, GMRES_GSflag=gs, **case)
    xh, xl, h, n, ir = oracle.ddcg(A, b, solver=3, **kw)
    _, h64, n64, ir64 = oracle.solve(A, b, solver=3, **kw)
    assert ir == ir64 == 0 and n == n64
    assert np.max(np.abs(h - h64) / h64) < 1e-5
    assert oracle.true_relres(A, b, xh + xl) < 1e-10


def test_ddgmres_itrmax_conventions():
    """niter = itr + inner at the itrmax stop (iret 0); itrmax = 1 runs one full cycle (iret 1)."""
    A, b = _system(10, 5)
    kw = dict(rtolmax=1e-15, GMRES_m=6, ipreflag=1)
    _, _, h, n, ir = oracle.ddcg(A, b, solver=3, itrmax=15, **kw)
    assert (n, ir, len(h)) == (15, 0, 15)
    xh, _, h, n, ir = oracle.ddcg(A, b, solver=3, itrmax=1, **kw)
    assert (n, ir, len(h)) == (1, 1, 1) and h[0] == 1.0
    assert oracle.true_relres(A, b, xh) < 1.0
