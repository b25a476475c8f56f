"""Pins the CPU oracle to the reference's stored outputs.

Known answers (src/example/template_cpu/STDOUT_run and template_gpu/STDOUT_run): CG on the
160^3 Poisson problem of src/example/problem.f90, rtolmax 1e-9, x0 = 0.
  * block-Jacobi D-ILU (ILU_method=1), 80 blocks: 291 iterations, rel. error 5.1459e-9;
  * block-Jacobi ILU(0), 4 blocks (cuSPARSE on GPU, one block per rank): 227 iterations;
  * double-double CG (template_cpu/STDOUT_run_dd, every PRECISION_* = 2), block-Jacobi
    D-ILU, 80 blocks: 291 iterations, max|x - x_exact| = 4.957113223374998e-9.
Match criteria: iteration count within +-2 and per-iteration relative history difference
<= 1e-6 (the reference's OpenMP/MPI reductions sum in a different order).
"""
import numpy as np
import pytest

from conftest import golden, poisson_reference
import oracle


def _check(case, **kw):
    fx = golden()[case]
    A, b, xe = poisson_reference(160)
    x, h, niter, iret = oracle.solve(A, b, solver=1, ipreflag=2, itrmax=2000, rtolmax=1e-9, **kw)
    g = np.array(fx["history_crs"])
    assert iret == 0
    assert abs(niter - len(g)) <= 2
    k = min(len(g), len(h))
    rel = np.abs(h[:k] - g[:k]) / g[:k]
    assert rel.max() <= 1e-6, rel.max()
    err = np.abs(x - xe).max() / np.abs(xe).max()
    assert abs(err - fx["rel_err"]) / fx["rel_err"] < 1e-3
    return niter, rel.max()


@pytest.mark.slow
def test_cg_dilu80_matches_template_cpu():
    niter, dev = _check("cpu_cg_dilu80", ILU_method=1, precon_thblock=80)
    assert niter == 291


@pytest.mark.slow
def test_cg_ilu0_4blocks_matches_template_gpu():
    niter, dev = _check("gpu_cg_ilu0_4", ILU_method=0, precon_thblock=4)
    assert niter == 227


def test_small_solvers_converge():
    """Every oracle solver reaches the tolerance on a small SPD problem."""
    A, b, xe = poisson_reference(10)
    for solver in (1, 2, 3):
        for pre in (dict(ipreflag=0), dict(ipreflag=1), dict(ipreflag=2, ILU_method=0, precon_thblock=3),
                    dict(ipreflag=2, ILU_method=1, precon_thblock=3), dict(ipreflag=2, ILU_method=2, precon_thblock=3)):
            x, h, niter, iret = oracle.solve(A, b, solver=solver, itrmax=500, rtolmax=1e-9, GMRES_m=20, **pre)
            assert iret == 0, (solver, pre)
            assert oracle.true_relres(A, b, x) < 1e-7, (solver, pre)


def test_oracle_matches_scipy_spmv():
    from parcel_b import problems
    A = problems.banded_random(5000, seed=3)
    x = np.random.default_rng(0).standard_normal(A.n)
    y = oracle.spmv(A, x)
    y2 = A.to_scipy() @ x
    assert np.allclose(y, y2, rtol=1e-13, atol=1e-13)


def test_oracle_ilu0_is_exact_for_tridiagonal():
    """ILU(0) of a tridiagonal block is its exact LU, so one application solves it."""
    import scipy.sparse as sp
    from parcel_b.problems import CRS
    n = 200
    rng = np.random.default_rng(1)
    M = sp.diags([rng.random(n - 1) - 0.5, 4 + rng.random(n), rng.random(n - 1) - 0.5], [-1, 0, 1]).tocsr()
    M.sort_indices()
    A = CRS(n=n, rowptr=(M.indptr + 1).astype(np.int32), col=(M.indices + 1).astype(np.int32), val=M.data.copy())
    r = rng.standard_normal(n)
    s = oracle.precon_apply(A, r, ipreflag=2, ILU_method=0, precon_thblock=1)
    assert np.allclose(M @ s, r, rtol=1e-12, atol=1e-12)


@pytest.mark.slow
def test_ddcg_dilu80_matches_template_cpu_dd():
    """The oracle's double-double CG (ddKSP_pCG) against STDOUT_run_dd's dd history."""
    fx = golden()["cpu_cg_dilu80_dd"]
    A, b, xe = poisson_reference(160)
    xh, xl, h, niter, iret = oracle.ddcg(A, b, ipreflag=2, ILU_method=1, precon_thblock=80, itrmax=2000,
                                         rtolmax=1e-9)
    g = np.array(fx["history_dd"])
    assert iret == 0 and abs(niter - len(g)) <= 2
    k = min(len(g), len(h))
    assert (np.abs(h[:k] - g[:k]) / g[:k]).max() <= 1e-6
    err = np.abs(xh + xl - xe).max()
    assert abs(err - fx["abs_err"]) / fx["abs_err"] < 1e-3
