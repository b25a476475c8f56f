"""The hot path's configurations at their stated sizes, GPU against the oracle.

  C1  PCG + point Jacobi, 2D 5-point Poisson 256^2, rtol 1e-8 (recursive residual)
  C2  PGMRES(30) MGS + block-Jacobi ILU(0) 64 blocks, 3D upwind convection-diffusion 128^3,
      rtol 1e-10 (the benchmark's drop-in workload)
  C3  mixed precision (FP32 PCG + FP32 block-Jacobi ILU(0) in FP64 / double-double
      refinement), anisotropic 7-point (1, 1e-2, 1e-4) 192^3, FP64 true residual 1e-12
  C4  CA-GMRES(s=8, t=8), Newton basis, TSQR, point Jacobi, random banded n = 4,000,000

Tolerances (the survey's parity criteria): iteration counts within +-2, residual
histories within 1e-6 relative while above 1e-8 of the first entry (before round-off
stagnation), true relative residuals at the tolerance.  For C3 the solution error against
the FP64 oracle's solution (solved to 1e-13) is bounded by 1e-7 relative: both solutions
have a true residual of at most 1e-12 and the matrix's condition number is about 1.5e4.
Against a double-double reference solve the bound is 1e-8 at 64^3 (condition about 1.7e3).
"""
import numpy as np
import pytest

import cagmres
import oracle
from parcel_b import api, problems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch
    assert torch.cuda.is_available()
    return torch


def _on(torch, A, b):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t(A.rowptr), t(A.col), t(A.val), t(b)


def _history_close(h, g, floor=1e-8):
    k = min(len(h), len(g))
    h, g = np.asarray(h[:k]), np.asarray(g[:k])
    m = g > floor * g[0]
    return float(np.max(np.abs(h[m] - g[m]) / g[m]))


def test_c2_gmres_convdiff128_matches_oracle(dev):
    A = problems.convdiff3d_upwind(128)
    b = problems.rhs_normal(A.n, 2)
    kw = dict(solver=3, ipreflag=2, ILU_method=0, precon_thblock=64, GMRES_m=30, GMRES_GSflag=1, itrmax=5000,
              rtolmax=1e-10)
    xo, ho, no, io = oracle.solve(A, b, **kw)
    rp, ci, va, bd = _on(dev, A, b)
    r = api.solve(A, bd, rowptr=rp, col=ci, val=va, **kw)
    assert r["iret"] == 0 and io == 0
    assert abs(r["niter"] - no) <= 2, (r["niter"], no)
    assert _history_close(r["reshistory"], ho) < 1e-6
    assert oracle.true_relres(A, b, r["x"].cpu().numpy()) <= 1.05e-10


def test_c1_pcg_poisson2d_256_matches_oracle(dev):
    A = problems.poisson2d_5pt(256, 256)
    b = problems.rhs_uniform(A.n, 1)
    kw = dict(solver=1, ipreflag=1, itrmax=5000, rtolmax=1e-8)
    xo, ho, no, io = oracle.solve(A, b, **kw)
    rp, ci, va, bd = _on(dev, A, b)
    r = api.solve(A, bd, rowptr=rp, col=ci, val=va, **kw)
    assert r["iret"] == 0 and io == 0
    assert abs(r["niter"] - no) <= 2, (r["niter"], no)
    assert _history_close(r["reshistory"], ho) < 1e-6
    x = r["x"].cpu().numpy()
    assert oracle.true_relres(A, b, x) < 2e-8
    assert np.max(np.abs(x - xo)) / np.max(np.abs(xo)) < 1e-6


def test_c3_mixed_aniso192_reaches_1e12_against_fp64_oracle(dev):
    A = problems.aniso3d(192, k=(1.0, 1e-2, 1e-4))
    b = problems.rhs_uniform(A.n, 3)
    rp, ci, va, bd = _on(dev, A, b)
    r = api.solve(A, bd, rowptr=rp, col=ci, val=va, solver=1, ipreflag=2, ILU_method=0, precon_thblock=64,
                  itrmax=20000, rtolmax=1e-12, inner_precision=1, residual_dd=1, inner_rtol=1e-4, max_refine=80)
    assert r["iret"] == 0, r["stats"]
    x = r["x"].cpu().numpy()
    assert oracle.true_relres(A, b, x) < 1e-12
    assert r["stats"]["true_relres_dd"] < 1e-12
    assert r["stats"]["refine_steps"] >= 2
    xo, ho, no, io = oracle.solve(A, b, solver=1, ipreflag=2, ILU_method=0, precon_thblock=64, itrmax=20000,
                                  rtolmax=1e-13)
    assert io == 0
    assert np.max(np.abs(x - xo)) / np.max(np.abs(xo)) < 1e-7


def test_c3_mixed_against_double_double_oracle(dev):
    A = problems.aniso3d(64, k=(1.0, 1e-2, 1e-4))
    b = problems.rhs_uniform(A.n, 3)
    rp, ci, va, bd = _on(dev, A, b)
    r = api.solve(A, bd, rowptr=rp, col=ci, val=va, solver=1, ipreflag=2, ILU_method=0, precon_thblock=64,
                  itrmax=20000, rtolmax=1e-12, inner_precision=1, residual_dd=1, inner_rtol=1e-4, max_refine=80)
    assert r["iret"] == 0
    x = r["x"].cpu().numpy()
    # the oracle's dd CG (D-ILU, 64 blocks) to a dd recursive residual of 1e-24
    xh, xl, h, n, i = oracle.ddcg(A, b, solver=1, ipreflag=2, ILU_method=1, precon_thblock=64, itrmax=20000,
                                  rtolmax=1e-24)
    assert i == 0
    err = np.max(np.abs((x - xh) - xl)) / np.max(np.abs(xh))
    assert err < 1e-8, err


def test_c4_cagmres_banded_4m_matches_oracle(dev):
    A = problems.banded_random(4_000_000, bandwidth=64, nnz_row=9, seed=4)
    b = problems.rhs_normal(A.n, 4)
    xo, ho, no, io = cagmres.pcagmres(A, b, s=8, t=8, basis=1, qrflag=3, itrmax=3000, rtolmax=1e-10, ipreflag=1)
    rp, ci, va, bd = _on(dev, A, b)
    r = api.solve(A, bd, rowptr=rp, col=ci, val=va, solver=4, CAGMRES_sstep=8, CAGMRES_tstep=8, CAGMRES_basis=1,
                  CAGMRES_QRflag=3, ipreflag=1, itrmax=3000, rtolmax=1e-10)
    assert r["iret"] == 0 and io == 0
    assert abs(r["niter"] - no) <= 2, (r["niter"], no)
    assert _history_close(r["reshistory"], ho) < 1e-6
    assert oracle.true_relres(A, b, r["x"].cpu().numpy()) < 2e-10
