"""Double-double PCG on the GPU (parcel_b_ddcg / parcel_ddcg_c_) against the oracle.

The GPU solve uses the reference's dd operation order (dd_func.f90), the reference's
per-row loop orders and the oracle's fixed dot-product split, so on the same inputs its
x (hi and lo), its residual history and its iteration count equal the oracle's bit for
bit.  At the reference's own configuration (template_cpu/STDOUT_run_dd: 160^3 Poisson,
block-Jacobi D-ILU with 80 blocks, every PRECISION_* = 2, rtol 1e-9) it also reproduces
the stored dd history (291 iterations) and the stored final error.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden, poisson_reference
import oracle

pytestmark = pytest.mark.gpu


def _gpu(A, b, **kw):
    from parcel_b import api
    return api.ddcg(A, b, **kw)


def _lo(v, seed):
    """Small low parts (below half an ulp of the high parts) to exercise dd inputs."""
    rng = np.random.default_rng(seed)
    return np.asarray(v) * 1e-17 * rng.uniform(-1.0, 1.0, len(v))


CASES = [
    dict(ipreflag=2, ILU_method=1, precon_thblock=8),
    dict(ipreflag=2, ILU_method=2, precon_thblock=5),
    dict(ipreflag=1),
    dict(ipreflag=0),
]


@pytest.mark.parametrize("case", CASES, ids=["dilu-ilud-8", "dilu-mlud-5", "point-jacobi", "none"])
def test_ddcg_matches_oracle_bit_for_bit(case):
    A, b, _ = poisson_reference(24)
    kw = dict(itrmax=400, rtolmax=1e-12, **case)
    g = _gpu(A, b, **kw)
    xh, xl, h, niter, iret = oracle.ddcg(A, b, **kw)
    assert g["iret"] == iret == 0
    assert g["niter"] == niter
    assert np.array_equal(g["reshistory"], h)
    assert np.array_equal(g["x_hi"], xh) and np.array_equal(g["x_lo"], xl)


@pytest.mark.parametrize("prec", [(1, 2, 2, 2), (2, 1, 2, 1), (2, 2, 1, 2)],
                         ids=["A-double", "b-double+M-double", "x-double"])
def test_ddcg_precision_flags_match_oracle(prec):
    pa, pb, px, pm = prec
    A, b, _ = poisson_reference(20)
    alo, blo = _lo(A.val, 1), _lo(b, 2)
    kw = dict(itrmax=300, rtolmax=1e-11, ipreflag=2, ILU_method=1, precon_thblock=4)
    g = _gpu(A, b, b_lo=blo, val_lo=alo, precision_A=pa, precision_b=pb, precision_x=px,
             precision_precondition=pm, **kw)
    xh, xl, h, niter, iret = oracle.ddcg(A, b, b_lo=blo, a_lo=alo, prec_A=pa, prec_b=pb, prec_x=px, prec_M=pm,
                                         **kw)
    assert g["niter"] == niter and g["iret"] == iret
    assert np.array_equal(g["reshistory"], h)
    assert np.array_equal(g["x_hi"], xh)
    if px == 2:
        assert np.array_equal(g["x_lo"], xl)


def test_ddcg_c_shim_matches_native_entry():
    """parcel_ddcg_c_ (the reference's argument order, host arrays) equals parcel_b_ddcg."""
    from parcel_b import _lib
    A, b, _ = poisson_reference(16)
    n = A.n
    ref = _gpu(A, b, itrmax=200, rtolmax=1e-10, ipreflag=2, ILU_method=1, precon_thblock=4)
    x, xl, blo = np.zeros(n), np.zeros(n), np.zeros(n)
    alo = np.zeros(A.nnz)
    hist = np.zeros(200)
    I = lambda v: C.byref(C.c_int(v))
    i32 = lambda v: C.byref(C.c_int32(v))
    niter, iret = C.c_int(200), C.c_int(0)
    ptr = lambda a: a.ctypes.data
    _lib.load().parcel_ddcg_c_(I(0), ptr(x), ptr(xl), ptr(b), ptr(blo), i32(n), i32(n), i32(A.nnz), i32(1),
                               ptr(A.val), ptr(alo), ptr(A.rowptr), ptr(A.col), I(2), I(1), I(0), I(1),
                               C.byref(niter), C.byref(C.c_double(1e-10)), ptr(hist), I(0), I(4), I(1), I(1),
                               I(2000), I(2), I(2), I(2), I(2), C.byref(iret))
    assert iret.value == 0 and niter.value == ref["niter"]
    assert np.array_equal(x, ref["x_hi"]) and np.array_equal(xl, ref["x_lo"])
    assert np.array_equal(hist[: niter.value], ref["reshistory"])


def test_ddcg_reproduces_reference_dd_output():
    """template_cpu/STDOUT_run_dd: 291 iterations, dd history, max|x - x_exact| = 4.957e-9."""
    fx = golden()["cpu_cg_dilu80_dd"]
    A, b, xe = poisson_reference(160)
    g = _gpu(A, b, itrmax=2000, rtolmax=1e-9, ipreflag=2, ILU_method=1, precon_thblock=80)
    ref = np.array(fx["history_dd"])
    assert g["iret"] == 0 and abs(g["niter"] - len(ref)) <= 2
    k = min(len(ref), len(g["reshistory"]))
    assert (np.abs(g["reshistory"][:k] - ref[:k]) / ref[:k]).max() <= 1e-6
    err = np.abs(g["x_hi"] + g["x_lo"] - xe).max()
    assert abs(err - fx["abs_err"]) / fx["abs_err"] < 1e-3


def _convdiff(g, seed):
    from parcel_b import problems
    A = problems.convdiff3d_upwind(g)
    return A, problems.rhs_normal(A.n, seed)


@pytest.mark.parametrize("case", CASES, ids=["dilu-ilud-8", "dilu-mlud-5", "point-jacobi", "none"])
def test_ddbicgstab_matches_oracle_bit_for_bit(case):
    """ddKSP_pBiCG on a nonsymmetric 3D convection-diffusion matrix."""
    from parcel_b import api
    A, b = _convdiff(20, 4)
    kw = dict(itrmax=400, rtolmax=1e-12, **case)
    g = api.ddbicgstab(A, b, **kw)
    xh, xl, h, niter, iret = oracle.ddcg(A, b, solver=2, **kw)
    assert g["iret"] == iret == 0
    assert g["niter"] == niter
    assert np.array_equal(g["reshistory"], h)
    assert np.array_equal(g["x_hi"], xh) and np.array_equal(g["x_lo"], xl)


def test_ddbicgstab_precision_flags_and_shim():
    """Mixed precision flags, and parcel_ddbicgstab_c_ against the native entry."""
    from parcel_b import _lib, api
    A, b = _convdiff(16, 5)
    alo, blo = _lo(A.val, 6), _lo(b, 7)
    kw = dict(itrmax=300, rtolmax=1e-11, ipreflag=2, ILU_method=1, precon_thblock=4)
    g = api.ddbicgstab(A, b, b_lo=blo, val_lo=alo, precision_A=2, precision_b=2, precision_x=2,
                       precision_precondition=1, **kw)
    xh, xl, h, niter, iret = oracle.ddcg(A, b, solver=2, b_lo=blo, a_lo=alo, prec_M=1, **kw)
    assert g["niter"] == niter and np.array_equal(g["reshistory"], h)
    assert np.array_equal(g["x_hi"], xh) and np.array_equal(g["x_lo"], xl)
    n = A.n
    x, xl2 = np.zeros(n), np.zeros(n)
    hist = np.zeros(300)
    I = lambda v: C.byref(C.c_int(v))
    i32 = lambda v: C.byref(C.c_int32(v))
    it, ir = C.c_int(300), C.c_int(0)
    ptr = lambda a: a.ctypes.data
    _lib.load().parcel_ddbicgstab_c_(I(0), ptr(x), ptr(xl2), ptr(b), ptr(blo), i32(n), i32(n), i32(A.nnz), i32(1),
                                     ptr(A.val), ptr(alo), ptr(A.rowptr), ptr(A.col), I(2), I(1), I(0), I(1),
                                     C.byref(it), C.byref(C.c_double(1e-11)), ptr(hist), I(0), I(4), I(1), I(1),
                                     I(2000), I(2), I(2), I(2), I(1), C.byref(ir))
    assert ir.value == 0 and it.value == niter
    assert np.array_equal(x, xh) and np.array_equal(xl2, xl)


GM_CASES = [
    dict(GMRES_GSflag=1, ipreflag=2, ILU_method=1, precon_thblock=8),
    dict(GMRES_GSflag=2, ipreflag=2, ILU_method=2, precon_thblock=5),
    dict(GMRES_GSflag=1, ipreflag=1),
    dict(GMRES_GSflag=2, ipreflag=0),
]


@pytest.mark.parametrize("case", GM_CASES, ids=["mgs-dilu-ilud-8", "cgs-dilu-mlud-5", "mgs-point-jacobi",
                                                "cgs-none"])
def test_ddgmres_matches_oracle_bit_for_bit(case):
    """ddKSP_pGMRES(10) on a nonsymmetric 3D convection-diffusion matrix, several restarts."""
    from parcel_b import api
    A, b = _convdiff(18, 8)
    kw = dict(itrmax=400, rtolmax=1e-12, GMRES_m=10, **case)
    g = api.ddgmres(A, b, **kw)
    xh, xl, h, niter, iret = oracle.ddcg(A, b, solver=3, **kw)
    assert g["iret"] == iret == 0
    assert g["niter"] == niter
    assert np.array_equal(g["reshistory"], h)
    assert np.array_equal(g["x_hi"], xh) and np.array_equal(g["x_lo"], xl)


@pytest.mark.parametrize("itrmax,want_iret", [(23, 0), (1, 1)], ids=["inside-a-cycle", "itrmax-1"])
def test_ddgmres_iteration_limit_and_precision_flags(itrmax, want_iret):
    """The reference's itrmax handling: the stop at itr + inner == itrmax keeps iret 0; with
    itrmax = 1 that stop cannot fire, the first cycle runs all m steps and iret is 1.  A and
    M in double, b and x in double-double."""
    from parcel_b import api
    A, b = _convdiff(14, 9)
    alo, blo = _lo(A.val, 10), _lo(b, 11)
    kw = dict(itrmax=itrmax, rtolmax=1e-14, GMRES_m=8, GMRES_GSflag=1, ipreflag=2, ILU_method=1,
              precon_thblock=4)
    g = api.ddgmres(A, b, b_lo=blo, val_lo=alo, precision_A=1, precision_b=2, precision_x=2,
                    precision_precondition=1, **kw)
    xh, xl, h, niter, iret = oracle.ddcg(A, b, solver=3, b_lo=blo, a_lo=alo, prec_A=1, prec_M=1, **kw)
    assert g["iret"] == iret == want_iret and g["niter"] == niter == itrmax
    assert np.array_equal(g["reshistory"], h)
    assert np.array_equal(g["x_hi"], xh) and np.array_equal(g["x_lo"], xl)


def test_ddgmres_c_shim_matches_native_entry():
    """parcel_ddgmres_c_ (restart and Gram-Schmidt flag after nblock) equals parcel_b_ddgmres."""
    from parcel_b import _lib, api
    A, b = _convdiff(12, 12)
    n = A.n
    ref = api.ddgmres(A, b, itrmax=300, rtolmax=1e-11, GMRES_m=12, GMRES_GSflag=2, ipreflag=2, ILU_method=1,
                      precon_thblock=4)
    x, xl, blo = np.zeros(n), np.zeros(n), np.zeros(n)
    alo = np.zeros(A.nnz)
    hist = np.zeros(300)
    I = lambda v: C.byref(C.c_int(v))
    i32 = lambda v: C.byref(C.c_int32(v))
    it, ir = C.c_int(300), C.c_int(0)
    ptr = lambda a: a.ctypes.data
    _lib.load().parcel_ddgmres_c_(I(0), ptr(x), ptr(xl), ptr(b), ptr(blo), i32(n), i32(n), i32(A.nnz), i32(1),
                                  ptr(A.val), ptr(alo), ptr(A.rowptr), ptr(A.col), I(2), I(1), I(0), I(1),
                                  C.byref(it), C.byref(C.c_double(1e-11)), ptr(hist), I(0), I(4), I(1), I(1),
                                  I(2000), I(12), I(2), I(2), I(2), I(2), I(2), C.byref(ir))
    assert ir.value == 0 and it.value == ref["niter"]
    assert np.array_equal(x, ref["x_hi"]) and np.array_equal(xl, ref["x_lo"])
    assert np.array_equal(hist[: it.value], ref["reshistory"])
