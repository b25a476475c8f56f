"""DIA input on the GPU (parcel_b_solve_dia, parcel_b_ddsolve_dia and the parcel_d*_dia_c_
shims) against the CRS path.

The DIA arrays are converted once, on the device, into the CRS matrix they stand for
(dia2crs, src/matrix.f90:7536-7576: the nonzero entries, here in ascending column order),
and the CRS solver runs on it.  The GPU solves are deterministic, so a DIA solve must
equal the CRS solve of the same matrix bit for bit; the reference's 160^3 template
(template_cpu/STDOUT_run, identical CRS and DIA histories) is reproduced through
parcel_dcg_dia_c_.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import golden, poisson_reference
from parcel_b import _lib, api, problems

pytestmark = pytest.mark.gpu

I = lambda v: C.byref(C.c_int(v))
i32 = lambda v: C.byref(C.c_int32(v))
ptr = lambda a: a.ctypes.data


def _scrambled_dia(A, seed=1):
    """The DIA arrays of A with the diagonals in a shuffled order."""
    dia, off = oracle.crs_to_dia(A)
    p = np.random.default_rng(seed).permutation(len(off))
    return np.ascontiguousarray(dia.reshape(len(off), A.n)[p].ravel()), np.ascontiguousarray(off[p])


SOLVES = [
    dict(solver=1, ipreflag=2, ILU_method=1, precon_thblock=6),
    dict(solver=2, ipreflag=2, ILU_method=0, precon_thblock=4),
    dict(solver=3, ipreflag=2, ILU_method=2, precon_thblock=3, GMRES_m=10, GMRES_GSflag=2),
    dict(solver=4, ipreflag=1, CAGMRES_sstep=4, CAGMRES_tstep=2, CAGMRES_basis=0, CAGMRES_QRflag=5),
    dict(solver=3, ipreflag=0, GMRES_m=20, GMRES_GSflag=1),
]


@pytest.mark.parametrize("kw", SOLVES, ids=lambda d: "-".join(f"{k}{v}" for k, v in d.items()))
def test_dia_solve_equals_crs_solve(kw):
    # CG on the symmetric Poisson matrix, the others on nonsymmetric convection-diffusion
    A = poisson_reference(14)[0] if kw["solver"] == 1 else problems.convdiff3d_upwind(14)
    b = np.random.default_rng(3).standard_normal(A.n)
    kw = dict(kw, itrmax=1000, rtolmax=1e-10)
    ref = api.solve(A, b, **kw)
    dia, off = _scrambled_dia(A)
    got = api.solve_dia(dia, off, b, **kw)
    assert ref["iret"] == got["iret"] == 0 and ref["niter"] == got["niter"]
    assert np.array_equal(ref["reshistory"], got["reshistory"])
    assert np.array_equal(ref["x"], got["x"])


def test_dia_device_arrays_equal_host_arrays():
    import torch
    A = problems.convdiff3d_upwind(12)
    b = np.random.default_rng(4).standard_normal(A.n)
    dia, off = _scrambled_dia(A, 2)
    kw = dict(solver=3, ipreflag=2, ILU_method=0, precon_thblock=8, GMRES_m=20, itrmax=500, rtolmax=1e-10)
    h = api.solve_dia(dia, off, b, **kw)
    t = lambda a: torch.from_numpy(a).cuda()
    d = api.solve_dia(t(dia), t(off), t(b), **kw)
    assert h["niter"] == d["niter"] and np.array_equal(h["reshistory"], d["reshistory"])
    assert np.array_equal(h["x"], d["x"].cpu().numpy())


def test_dia_out_of_range_entries_are_left_out():
    A = problems.convdiff3d_upwind(10)
    b = np.random.default_rng(5).standard_normal(A.n)
    dia, off = oracle.crs_to_dia(A)
    d = dia.reshape(len(off), A.n).copy()
    d[int(np.argmin(off)), 0] = 5.0            # column before row 1
    d[int(np.argmax(off)), A.n - 1] = -2.0     # column after row n
    kw = dict(solver=2, ipreflag=1, itrmax=500, rtolmax=1e-10)
    ref = api.solve(A, b, **kw)
    got = api.solve_dia(np.ascontiguousarray(d.ravel()), off, b, **kw)
    assert ref["niter"] == got["niter"] and np.array_equal(ref["x"], got["x"])


def test_dia_repeated_offset_is_an_error():
    A = problems.convdiff3d_upwind(6)
    dia, off = oracle.crs_to_dia(A)
    off2 = off.copy()
    off2[1] = off2[0]
    with pytest.raises(RuntimeError, match="appears twice"):
        api.solve_dia(dia, off2, np.ones(A.n), solver=1, itrmax=10)


def test_fp64_dia_shims_equal_crs_shims():
    A = poisson_reference(11)[0]
    b = np.random.default_rng(6).standard_normal(A.n)
    n = A.n
    dia, off = _scrambled_dia(A, 3)
    L = _lib.load()
    common_crs = lambda x, h, it, ir: (I(0), ptr(x), ptr(b), i32(n), i32(n), i32(A.nnz), i32(1), ptr(A.val),
                                       ptr(A.rowptr), ptr(A.col), I(2), I(0), I(0), I(1), C.byref(it),
                                       C.byref(C.c_double(1e-10)), ptr(h), I(0), I(4), I(1), I(1), I(2000))
    common_dia = lambda x, h, it, ir: (I(0), ptr(x), ptr(b), i32(n), i32(n), i32(1), ptr(dia), ptr(off),
                                       i32(len(off)), I(2), I(0), I(0), I(1), C.byref(it),
                                       C.byref(C.c_double(1e-10)), ptr(h), I(0), I(4), I(1), I(1), I(2000))
    for crs_fn, dia_fn, extra in [
        (L.parcel_dcg_c_, L.parcel_dcg_dia_c_, ()),
        (L.parcel_dbicgstab_c_, L.parcel_dbicgstab_dia_c_, ()),
        (L.parcel_dgmres_c_, L.parcel_dgmres_dia_c_, (I(15), I(1))),
        (L.parcel_dcagmres_c_, L.parcel_dcagmres_dia_c_, (I(4), I(4), I(0), I(3))),
    ]:
        out = []
        for fn, common in ((crs_fn, common_crs), (dia_fn, common_dia)):
            x, h = np.zeros(n), np.zeros(500)
            it, ir = C.c_int(500), C.c_int(0)
            fn(*common(x, h, it, ir), *extra, C.byref(ir))
            out.append((x, h[: it.value].copy(), it.value, ir.value))
        (x1, h1, n1, r1), (x2, h2, n2, r2) = out
        assert r1 == r2 == 0 and n1 == n2, dia_fn
        assert np.array_equal(h1, h2) and np.array_equal(x1, x2), dia_fn


@pytest.mark.parametrize("solver", [1, 2, 3], ids=["ddcg", "ddbicgstab", "ddgmres"])
def test_dd_dia_equals_dd_crs(solver):
    A = poisson_reference(10)[0]
    b = np.random.default_rng(7).standard_normal(A.n)
    alo = A.val * 1e-17 * np.random.default_rng(8).uniform(-1, 1, A.nnz)
    blo = b * 1e-17
    dia, off = oracle.crs_to_dia(A)
    dlo, _ = oracle.crs_to_dia(A, val=alo)
    kw = dict(itrmax=400, rtolmax=1e-12, ipreflag=2, ILU_method=1, precon_thblock=4, GMRES_m=12)
    ref = api.ddcg(A, b, b_lo=blo, val_lo=alo, solver=solver, **kw)
    got = api.ddsolve_dia(dia, off, b, b_lo=blo, val_lo=dlo, solver=solver, **kw)
    assert ref["iret"] == got["iret"] == 0 and ref["niter"] == got["niter"]
    assert np.array_equal(ref["reshistory"], got["reshistory"])
    assert np.array_equal(ref["x_hi"], got["x_hi"]) and np.array_equal(ref["x_lo"], got["x_lo"])


def test_dd_dia_shims_equal_dd_crs_shims():
    A = poisson_reference(9)[0]
    b = np.random.default_rng(9).standard_normal(A.n)
    n = A.n
    dia, off = oracle.crs_to_dia(A)
    zl, zd = np.zeros(A.nnz), np.zeros(dia.shape[0])
    L = _lib.load()
    for crs_fn, dia_fn, gm in [(L.parcel_ddcg_c_, L.parcel_ddcg_dia_c_, False),
                               (L.parcel_ddbicgstab_c_, L.parcel_ddbicgstab_dia_c_, False),
                               (L.parcel_ddgmres_c_, L.parcel_ddgmres_dia_c_, True)]:
        res = []
        for which in ("crs", "dia"):
            x, xl, bl, h = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(300)
            it, ir = C.c_int(300), C.c_int(0)
            head = (I(0), ptr(x), ptr(xl), ptr(b), ptr(bl))
            mat = ((i32(n), i32(n), i32(A.nnz), i32(1), ptr(A.val), ptr(zl), ptr(A.rowptr), ptr(A.col))
                   if which == "crs" else (i32(n), i32(n), i32(1), ptr(dia), ptr(zd), ptr(off), i32(len(off))))
            mid = (I(2), I(1), I(0), I(1), C.byref(it), C.byref(C.c_double(1e-11)), ptr(h), I(0), I(4))
            # parcel_ddgmres_dia_c_ has no Neuman_itr; the CRS dd shims all have it
            tail = (I(1), I(1), I(2000)) if (which == "crs" or not gm) else (I(1), I(2000))
            if gm:
                tail = tail + (I(10), I(1))
            fn = crs_fn if which == "crs" else dia_fn
            fn(*head, *mat, *mid, *tail, I(2), I(2), I(2), I(2), C.byref(ir))
            res.append((x, xl, h[: it.value].copy(), it.value, ir.value))
        (x1, l1, h1, n1, r1), (x2, l2, h2, n2, r2) = res
        assert r1 == r2 == 0 and n1 == n2, dia_fn
        assert np.array_equal(h1, h2) and np.array_equal(x1, x2) and np.array_equal(l1, l2), dia_fn


def test_reference_template_through_dia_shim():
    """template_cpu/STDOUT_run's DIA column: 160^3 CG + D-ILU, 80 blocks, through parcel_dcg_dia_c_."""
    fx = golden()["cpu_cg_dilu80"]
    A, b, xe = poisson_reference(160)
    dia, off = oracle.crs_to_dia(A)
    x = np.zeros(A.n)
    hist = np.zeros(2000)
    it, ir = C.c_int(2000), C.c_int(0)
    _lib.load().parcel_dcg_dia_c_(I(0), ptr(x), ptr(b), i32(A.n), i32(A.n), i32(1), ptr(dia), ptr(off),
                                  i32(len(off)), I(2), I(1), I(0), I(1), C.byref(it), C.byref(C.c_double(1e-9)),
                                  ptr(hist), I(0), I(80), I(1), I(1), I(2000), C.byref(ir))
    g = np.array(fx["history_crs"])
    assert ir.value == 0 and abs(it.value - len(g)) <= 2
    k = min(it.value, len(g))
    assert np.max(np.abs(hist[:k] - g[:k]) / g[:k]) < 1e-6
    err = np.abs(x - xe).max() / np.abs(xe).max()
    assert abs(err - fx["rel_err"]) / fx["rel_err"] < 1e-2
