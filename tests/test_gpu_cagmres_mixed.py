"""GPU CA-GMRES, mixed-precision refinement and the double-double residual against the
oracles.  Tolerances: residual histories within 1e-6 relative before stagnation,
iteration counts within +-2; the double-double residual within 4 dd ulps of the numpy
dd oracle (the kernel uses the reference's operation order, so it is usually exact)."""
import ctypes as C

import numpy as np
import pytest

import cagmres
import dd
import oracle
from parcel_b import _lib, api, problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("s,t,basis,qr,pre", [
    (4, 1, 0, 4, dict(ipreflag=1)),
    (4, 2, 0, 5, dict(ipreflag=1)),
    (2, 4, 0, 3, dict(ipreflag=2, ILU_method=0, precon_thblock=4)),
    (4, 3, 1, 5, dict(ipreflag=1)),
    (8, 4, 1, 3, dict(ipreflag=1)),
])
def test_gpu_cagmres_matches_oracle(s, t, basis, qr, pre):
    A = problems.convdiff3d_upwind(11)
    b = problems.rhs_normal(A.n, 3)
    xo, ho, no, io = cagmres.pcagmres(A, b, s=s, t=t, basis=basis, qrflag=qr, itrmax=800, rtolmax=1e-10, **pre)
    res = api.solve(A, b, solver=4, CAGMRES_sstep=s, CAGMRES_tstep=t, CAGMRES_basis=basis, CAGMRES_QRflag=qr,
                    itrmax=800, rtolmax=1e-10, **pre)
    assert res["iret"] == 0 and io == 0
    assert abs(res["niter"] - no) <= 2, (res["niter"], no)
    k = min(len(ho), len(res["reshistory"]))
    h, g = res["reshistory"][:k], ho[:k]
    m = g > 1e-8
    assert np.max(np.abs(h[m] - g[m]) / g[m]) < 1e-6
    assert oracle.true_relres(A, b, res["x"]) < 1e-9


def test_gpu_cagmres_banded_newton_tsqr():
    """The banded random nonsymmetric matrix of the CA-GMRES benchmark configuration, small."""
    A = problems.banded_random(20000, seed=11)
    b = problems.rhs_normal(A.n, 4)
    res = api.solve(A, b, solver=4, CAGMRES_sstep=8, CAGMRES_tstep=8, CAGMRES_basis=1, CAGMRES_QRflag=3,
                    ipreflag=1, itrmax=2000, rtolmax=1e-10)
    xg, hg, ng, ig = oracle.solve(A, b, solver=3, GMRES_m=64, GMRES_GSflag=1, ipreflag=1, itrmax=2000, rtolmax=1e-10)
    assert res["iret"] == 0
    assert abs(res["niter"] - ng) <= 2
    assert oracle.true_relres(A, b, res["x"]) < 1e-9


def test_residual_dd_matches_numpy_oracle():
    import torch
    A = problems.aniso3d(10)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(A.n)
    b = rng.standard_normal(A.n)
    rh_ref, rl_ref = dd.residual(A, x, None, b, None)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    rh, rl = torch.zeros(A.n, dtype=torch.float64, device="cuda"), torch.zeros(A.n, dtype=torch.float64, device="cuda")
    # the device copies must outlive the call: the struct holds raw pointers only
    rp, ci, va = t(A.rowptr), t(A.col), t(A.val)
    S = api.crs_struct(A, rp, ci, va)
    xd, bd = t(x), t(b)
    rc = _lib.load().parcel_b_residual_dd(C.byref(S), xd.data_ptr(), None, bd.data_ptr(), None, rh.data_ptr(),
                                          rl.data_ptr())
    assert rc == 0
    hi, lo = rh.cpu().numpy(), rl.cpu().numpy()
    err = np.abs((hi - rh_ref) + (lo - rl_ref))
    scale = np.abs(rh_ref) + 1e-300
    assert np.max(err / scale) < 4 * 2.0 ** -104


def test_mixed_precision_reaches_1e12():
    A = problems.aniso3d(14, k=(1.0, 1e-2, 1e-4))
    b = problems.rhs_uniform(A.n, 6)
    res = api.solve(A, b, solver=1, ipreflag=2, ILU_method=0, precon_thblock=7, itrmax=4000, rtolmax=1e-12,
                    inner_precision=1, residual_dd=1, inner_rtol=1e-4, max_refine=40)
    assert res["iret"] == 0, res["stats"]
    assert oracle.true_relres(A, b, res["x"]) < 1e-12
    assert res["stats"]["true_relres_dd"] < 1e-12
    assert res["stats"]["refine_steps"] >= 2
    # agrees with the FP64 oracle solution to the accuracy the tolerance allows
    xo, ho, no, io = oracle.solve(A, b, solver=1, ipreflag=2, ILU_method=0, precon_thblock=7, itrmax=4000,
                                  rtolmax=1e-13)
    assert np.max(np.abs(res["x"] - xo)) / np.max(np.abs(xo)) < 1e-8
