"""GPU parity: libparcelb (through its C-ABI) against the CPU oracle on the same inputs.

Tolerances (FP64): kernel outputs within 1e-12 relative (the GPU contracts a*b+c into FMA
and sums in a different order); solver residual histories within 1e-6 relative before
stagnation and iteration counts within +-2 of the oracle (the criteria the oracle itself
meets against the reference's stored output).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import golden, poisson_reference
from parcel_b import _lib, api, problems

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


MATS = {
    "poisson3d_12": lambda: poisson_reference(12)[0],
    "convdiff_10": lambda: problems.convdiff3d_upwind(10),
    "aniso_9": lambda: problems.aniso3d(9),
    "banded_3000": lambda: problems.banded_random(3000, seed=7),
    "poisson2d_40": lambda: problems.poisson2d_5pt(40, 40),
}


@pytest.mark.parametrize("name", list(MATS))
def test_spmv_matches_oracle(torch_cuda, name):
    torch = torch_cuda
    A = MATS[name]()
    x = np.random.default_rng(1).standard_normal(A.n)
    y_ref = oracle.spmv(A, x)
    rp, ci, va, xd = _dev(torch, A.rowptr), _dev(torch, A.col), _dev(torch, A.val), _dev(torch, x)
    yd = torch.zeros_like(xd)
    S = api.crs_struct(A, rp, ci, va)
    assert _lib.load().parcel_b_spmv(C.byref(S), xd.data_ptr(), yd.data_ptr()) == 0
    assert _rel(yd.cpu().numpy(), y_ref) < 1e-13


PRECONS = [
    dict(ipreflag=1),
    dict(ipreflag=2, ILU_method=0, precon_thblock=1),
    dict(ipreflag=2, ILU_method=0, precon_thblock=5),
    dict(ipreflag=2, ILU_method=1, precon_thblock=4),
    dict(ipreflag=2, ILU_method=2, precon_thblock=3),
    dict(ipreflag=3, ILU_method=0, precon_thblock=2),
]


@pytest.mark.parametrize("name", ["poisson3d_12", "convdiff_10", "banded_3000", "poisson2d_40"])
@pytest.mark.parametrize("pre", PRECONS, ids=lambda d: "-".join(f"{k}{v}" for k, v in d.items()))
def test_precon_matches_oracle(name, pre):
    A = MATS[name]()
    r = np.random.default_rng(2).standard_normal(A.n)
    s_ref = oracle.precon_apply(A, r, **pre)
    s = np.zeros(A.n)
    p = _lib.new_input(**pre)
    rc = _lib.load().parcel_b_precon_apply(C.byref(p), C.byref(api.crs_struct(A)), r.ctypes.data, s.ctypes.data)
    assert rc == 0, _lib.last_error()
    assert _rel(s, s_ref) < 1e-11


def _solve_both(A, b, **kw):
    xo, ho, no, io = oracle.solve(A, b, **kw)
    okw = dict(kw)
    res = api.solve(A, b, **okw)
    return (xo, ho, no, io), res


SOLVES = [
    ("poisson3d_12", dict(solver=1, ipreflag=0)),
    ("poisson3d_12", dict(solver=1, ipreflag=1)),
    ("poisson3d_12", dict(solver=1, ipreflag=2, ILU_method=1, precon_thblock=6)),
    ("poisson3d_12", dict(solver=1, ipreflag=2, ILU_method=0, precon_thblock=3)),
    ("poisson3d_12", dict(solver=2, ipreflag=2, ILU_method=0, precon_thblock=4)),
    ("convdiff_10", dict(solver=2, ipreflag=1)),
    ("convdiff_10", dict(solver=3, ipreflag=2, ILU_method=0, precon_thblock=4, GMRES_m=10, GMRES_GSflag=1)),
    ("convdiff_10", dict(solver=3, ipreflag=2, ILU_method=2, precon_thblock=2, GMRES_m=7, GMRES_GSflag=2)),
    ("banded_3000", dict(solver=3, ipreflag=1, GMRES_m=30, GMRES_GSflag=1)),
    ("banded_3000", dict(solver=2, ipreflag=0)),
    ("poisson2d_40", dict(solver=1, ipreflag=1)),
]


@pytest.mark.parametrize("name,kw", SOLVES, ids=[f"{n}-" + "-".join(f"{k}{v}" for k, v in d.items()) for n, d in SOLVES])
def test_solver_matches_oracle(name, kw):
    A = MATS[name]()
    b = np.random.default_rng(3).standard_normal(A.n)
    kw = dict(kw, itrmax=2000, rtolmax=1e-10)
    (xo, ho, no, io), res = _solve_both(A, b, **kw)
    assert io == 0 and res["iret"] == 0
    assert abs(res["niter"] - no) <= 2, (res["niter"], no)
    k = min(len(ho), len(res["reshistory"]))
    h, g = res["reshistory"][:k], ho[:k]
    m = g > 1e-8   # before stagnation
    assert np.all(np.abs(h[m] - g[m]) / g[m] < 1e-6), np.max(np.abs(h[m] - g[m]) / g[m])
    assert oracle.true_relres(A, b, res["x"]) < 1e-9
    assert _rel(res["x"], xo) < 1e-7


@pytest.mark.parametrize("case,kw", [
    ("cpu_cg_dilu80", dict(ILU_method=1, precon_thblock=80)),
    ("gpu_cg_ilu0_4", dict(ILU_method=0, precon_thblock=4)),
])
def test_reference_template_through_c_abi(case, kw):
    """The reference's 160^3 CG templates, solved through parcel_dcg_c_ with host arrays."""
    fx = golden()[case]
    A, b, xe = poisson_reference(160)
    x = np.zeros(A.n)
    hist = np.zeros(2000)
    niter, iret = api.parcel_dcg(x, b, A.n, A.n, A.nnz, 1, A.val, A.rowptr, A.col, 2, kw["ILU_method"],
                                 0, 1, 2000, 1e-9, hist, precon_thblock=kw["precon_thblock"])
    g = np.array(fx["history_crs"])
    assert iret == 0
    assert abs(niter - len(g)) <= 2
    k = min(niter, len(g))
    assert np.max(np.abs(hist[:k] - g[:k]) / g[:k]) < 1e-6
    err = np.abs(x - xe).max() / np.abs(xe).max()
    assert abs(err - fx["rel_err"]) / fx["rel_err"] < 1e-2


def test_gpu_abi_device_pointers_match_host(torch_cuda):
    torch = torch_cuda
    A = problems.convdiff3d_upwind(12)
    b = np.random.default_rng(4).standard_normal(A.n)
    x_h = np.zeros(A.n)
    h_h = np.zeros(500)
    n1, i1 = api.parcel_dgmres(x_h, b, A.n, A.n, A.nnz, 1, A.val, A.rowptr, A.col, 2, 0, 0, 1, 500, 1e-10,
                               h_h, precon_thblock=8, GMRES_m=20, GMRES_GSflag=1)
    x_d = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    h_d = np.zeros(500)
    n2, i2 = api.parcel_dgmres(x_d, _dev(torch, b), A.n, A.n, A.nnz, 1, _dev(torch, A.val), _dev(torch, A.rowptr),
                               _dev(torch, A.col), 2, 0, 0, 1, 500, 1e-10, h_d, precon_thblock=8, GMRES_m=20,
                               GMRES_GSflag=1)
    assert (n1, i1) == (n2, i2)
    assert np.array_equal(h_h[:n1], h_d[:n2])
    assert np.array_equal(x_h, x_d.cpu().numpy())


def test_deterministic_repeat():
    A = problems.convdiff3d_upwind(14)
    b = np.random.default_rng(5).standard_normal(A.n)
    r1 = api.solve(A, b, solver=3, ipreflag=2, ILU_method=0, precon_thblock=16, GMRES_m=30, itrmax=400, rtolmax=1e-10)
    r2 = api.solve(A, b, solver=3, ipreflag=2, ILU_method=0, precon_thblock=16, GMRES_m=30, itrmax=400, rtolmax=1e-10)
    assert np.array_equal(r1["x"], r2["x"]) and np.array_equal(r1["reshistory"], r2["reshistory"])


def test_maxiter_and_history_length():
    A = problems.convdiff3d_upwind(10)
    b = np.random.default_rng(6).standard_normal(A.n)
    for kw in (dict(solver=1, ipreflag=1), dict(solver=2, ipreflag=1), dict(solver=3, ipreflag=1, GMRES_m=4)):
        xo, ho, no, io = oracle.solve(A, b, itrmax=7, rtolmax=1e-14, **kw)
        res = api.solve(A, b, itrmax=7, rtolmax=1e-14, **kw)
        assert (res["niter"], res["iret"]) == (no, io), (kw, res["niter"], res["iret"], no, io)


def test_zero_pivot_is_an_error_not_a_crash():
    A = problems.poisson2d_5pt(6, 6)
    val = A.val.copy()
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    diag = (A.col - 1) == rows
    # drop row 5's diagonal entry structurally: keep CRS valid, remove the entry
    keep = ~(diag & (rows == 5))
    rp = np.concatenate([[1], 1 + np.cumsum(np.bincount(rows[keep], minlength=A.n))]).astype(np.int32)
    B = problems.CRS(n=A.n, rowptr=rp, col=A.col[keep].copy(), val=val[keep].copy())
    b = np.ones(A.n)
    with pytest.raises(RuntimeError, match=r"\[-1\]"):
        api.solve(B, b, solver=1, ipreflag=2, ILU_method=0, precon_thblock=2, itrmax=10, rtolmax=1e-8)


def test_multiprocess_layout_is_rejected():
    A = problems.poisson2d_5pt(8, 8)
    S = api.crs_struct(A)
    S.gn = A.n * 2
    p = _lib.new_input(solver=1, ipreflag=0, itrmax=5, rtolmax=1e-8)
    b = np.ones(A.n)
    x = np.zeros(A.n)
    niter, iret = C.c_int(0), C.c_int(0)
    rc = _lib.load().parcel_b_solve(C.byref(p), C.byref(S), b.ctypes.data, x.ctypes.data, None,
                                    C.byref(niter), C.byref(iret))
    assert rc == _lib.E_UNSUPPORTED and iret.value == _lib.E_UNSUPPORTED


def test_streaming_mgs_matches_oracle():
    """140^3 rows exceed what the register-resident fused MGS holds (32 elements per
    thread of the co-resident grid), so the streaming fused MGS runs; two restart cycles
    of its GMRES history must match the oracle's MGS GMRES."""
    A = problems.convdiff3d_upwind(140)
    b = problems.rhs_normal(A.n, 5)
    kw = dict(solver=3, ipreflag=2, ILU_method=0, precon_thblock=64, GMRES_m=30, GMRES_GSflag=1, itrmax=60,
              rtolmax=1e-12)
    res = api.solve(A, b, **kw)
    xo, ho, no, io = oracle.solve(A, b, **kw)
    assert res["niter"] == no == 60
    h = res["reshistory"]
    assert np.max(np.abs(h - ho) / ho) < 1e-6
    assert _rel(res["x"], xo) < 1e-6


@pytest.mark.parametrize("blocks", [1, 2])
@pytest.mark.parametrize("ilu", [0, 1])
def test_wide_levels_precon_matches_oracle(blocks, ilu):
    """Wavefronts wider than one row per consumer thread (up to 700 rows per level: 2, 4
    rows per thread) take the multi-row fast sweep."""
    A = problems.poisson2d_5pt(700, 700)
    pre = dict(ipreflag=2, ILU_method=ilu, precon_thblock=blocks)
    r = np.random.default_rng(3).standard_normal(A.n)
    s_ref = oracle.precon_apply(A, r, **pre)
    s = np.zeros(A.n)
    p = _lib.new_input(**pre)
    rc = _lib.load().parcel_b_precon_apply(C.byref(p), C.byref(api.crs_struct(A)), r.ctypes.data, s.ctypes.data)
    assert rc == 0, _lib.last_error()
    assert _rel(s, s_ref) < 1e-11


@pytest.mark.parametrize("ilu", [0, 1, 2])
@pytest.mark.parametrize("blocks", [2000, 5000])
def test_many_small_blocks_precon_matches_oracle(blocks, ilu):
    """Thousands of blocks of a few rows each (more than eight per SM, at most 1024 rows)
    take the warp-per-block sweep; uneven blocks (divide_region) and a nonsymmetric matrix."""
    A = problems.convdiff3d_upwind(24)
    pre = dict(ipreflag=2, ILU_method=ilu, precon_thblock=blocks)
    r = np.random.default_rng(4).standard_normal(A.n)
    s_ref = oracle.precon_apply(A, r, **pre)
    s = np.zeros(A.n)
    p = _lib.new_input(**pre)
    rc = _lib.load().parcel_b_precon_apply(C.byref(p), C.byref(api.crs_struct(A)), r.ctypes.data, s.ctypes.data)
    assert rc == 0, _lib.last_error()
    assert _rel(s, s_ref) < 1e-11
    # and a solve through it
    b = problems.rhs_normal(A.n, 6)
    kw = dict(solver=3, itrmax=2000, rtolmax=1e-10, GMRES_m=20, GMRES_GSflag=1, **pre)
    (xo, ho, no, io), res = _solve_both(A, b, **kw)
    assert io == 0 and res["iret"] == 0 and abs(res["niter"] - no) <= 2
    k = min(len(ho), len(res["reshistory"]))
    m = ho[:k] > 1e-8
    assert np.all(np.abs(res["reshistory"][:k][m] - ho[:k][m]) / ho[:k][m] < 1e-6)


@pytest.mark.parametrize("ilu", [0, 1])
def test_small_block_sweeps_staged_and_unstaged_match_oracle(ilu):
    """Many small blocks take one of two warp-per-block sweeps: a block whose stretch of the
    iteration layout (records, factors and right-hand side) fits 12 KB of shared memory per
    warp is staged there; longer ones read global memory.  On 64^3 rows, 1,200 blocks of about
    218 rows (66 levels, each padded to 4 positions) take the second, 20,000 blocks of
    about 13 rows the first; both against the oracle.  And the FP32 inner sweep of the
    mixed-precision solve through the staged one."""
    A = problems.convdiff3d_upwind(64)
    r = np.random.default_rng(7).standard_normal(A.n)
    for blocks in (1200, 20000):
        pre = dict(ipreflag=2, ILU_method=ilu, precon_thblock=blocks)
        s_ref = oracle.precon_apply(A, r, **pre)
        s = np.zeros(A.n)
        p = _lib.new_input(**pre)
        rc = _lib.load().parcel_b_precon_apply(C.byref(p), C.byref(api.crs_struct(A)), r.ctypes.data, s.ctypes.data)
        assert rc == 0, _lib.last_error()
        assert _rel(s, s_ref) < 1e-11, blocks
    P, bp, _ = problems.poisson3d_reference(24, 24, 24)
    res = api.solve(P, bp, solver=1, ipreflag=2, ILU_method=ilu, precon_thblock=2000, itrmax=4000, rtolmax=1e-12,
                    inner_precision=1, residual_dd=1, inner_rtol=1e-4, max_refine=40)
    assert res["iret"] == 0, res["stats"]
    assert oracle.true_relres(P, bp, res["x"]) < 1e-12


def test_diagonal_copy_spmv_path_matches_oracle():
    """Point Jacobi keeps the natural layout, where a stencil matrix's product runs on its
    diagonal copy (statistics: spmv_diagonals); CG and GMRES histories against the oracle at
    the parity criteria, and the banded random matrix (entries off any common diagonal set)
    stays on sliced ELLPACK."""
    import torch
    A = problems.convdiff3d_upwind(24)
    b = problems.rhs_normal(A.n, 5)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    kw = dict(solver=3, ipreflag=1, GMRES_m=30, itrmax=2000, rtolmax=1e-10)
    r = api.solve(A, t(b), rowptr=t(A.rowptr), col=t(A.col), val=t(A.val), **kw)
    assert r["stats"]["spmv_diagonals"] == 7
    xo, ho, no, io = oracle.solve(A, b, **kw)
    assert r["iret"] == io == 0 and abs(r["niter"] - no) <= 2
    k = min(len(ho), len(r["reshistory"]))
    m = ho[:k] > 1e-8 * ho[0]
    assert np.max(np.abs(np.asarray(r["reshistory"])[:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6
    P, bp, _ = problems.poisson3d_reference(20, 20, 20)
    r = api.solve(P, t(bp), rowptr=t(P.rowptr), col=t(P.col), val=t(P.val), solver=1, ipreflag=1, itrmax=2000,
                  rtolmax=1e-9)
    assert r["stats"]["spmv_diagonals"] == 7
    xo, ho, no, io = oracle.solve(P, bp, solver=1, ipreflag=1, itrmax=2000, rtolmax=1e-9)
    assert r["iret"] == io and abs(r["niter"] - no) <= 2
    B = problems.banded_random(20000, bandwidth=64, nnz_row=9, seed=4)
    bb = problems.rhs_normal(B.n, 4)
    r = api.solve(B, t(bb), rowptr=t(B.rowptr), col=t(B.col), val=t(B.val), solver=3, ipreflag=1, GMRES_m=30,
                  itrmax=500, rtolmax=1e-10)
    assert r["stats"]["spmv_diagonals"] == 0 and r["iret"] == 0
