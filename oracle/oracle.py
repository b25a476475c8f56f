"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py, always as the checker or the timed CPU reference, never as the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")


class OrcMat(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_int), ("istart", C.c_int),
                ("rowptr", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p)]


class OrcParams(C.Structure):
    _fields_ = [("solver", C.c_int), ("ipreflag", C.c_int), ("ILU_method", C.c_int),
                ("precon_thblock", C.c_int), ("itrmax", C.c_int), ("rtolmax", C.c_double),
                ("GMRES_m", C.c_int), ("GMRES_GSflag", C.c_int),
                ("CAGMRES_sstep", C.c_int), ("CAGMRES_tstep", C.c_int),
                ("CAGMRES_basis", C.c_int), ("CAGMRES_QRflag", C.c_int)]


def build(force: bool = False) -> str:
    if force or not os.path.exists(_LIB) or (
            os.path.getmtime(_LIB) < os.path.getmtime(os.path.join(_HERE, "parcel_oracle.cpp"))):
        subprocess.run(["make", "-C", _HERE, "-s", "-B" if force else "liboracle.so"], check=True)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.orc_solve.argtypes = [C.POINTER(OrcMat), C.POINTER(OrcParams), C.c_void_p, C.c_void_p,
                                C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_solve.restype = C.c_int
        L.orc_spmv.argtypes = [C.POINTER(OrcMat), C.c_void_p, C.c_void_p]
        L.orc_dot.argtypes = [C.c_long, C.c_void_p, C.c_void_p]
        L.orc_dot.restype = C.c_double
        L.orc_precon_apply.argtypes = [C.POINTER(OrcMat), C.POINTER(OrcParams), C.c_void_p, C.c_void_p]
        L.orc_precon_apply.restype = C.c_int
        L.orc_precon_dinv.argtypes = [C.POINTER(OrcMat), C.POINTER(OrcParams), C.c_void_p]
        L.orc_precon_dinv.restype = C.c_int
        L.orc_true_relres.argtypes = [C.POINTER(OrcMat), C.c_void_p, C.c_void_p]
        L.orc_true_relres.restype = C.c_double
        L.orc_num_threads.restype = C.c_int
        L.orc_precon_create.argtypes = [C.POINTER(OrcMat), C.POINTER(OrcParams), C.POINTER(C.c_int)]
        L.orc_precon_create.restype = C.c_void_p
        L.orc_precon_apply_h.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_precon_destroy.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_ddcg.argtypes = [C.POINTER(OrcMat), C.c_void_p, C.POINTER(OrcParams), C.c_int, C.c_int,
                               C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_ddcg.restype = C.c_int
        L.orc_set_blocks.argtypes = [C.c_int, C.c_void_p]
        L.orc_set_blocks.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class _Blocks:
    """Explicit block-Jacobi blocks for the calls inside the with-statement: `starts` are
    the 0-based first rows of the blocks followed by n (None: the equal split of
    precon_thblock)."""

    def __init__(self, starts):
        self.starts = None if starts is None else np.ascontiguousarray(starts, dtype=np.int64)

    def __enter__(self):
        if self.starts is not None:
            rc = lib().orc_set_blocks(len(self.starts) - 1, _ptr(self.starts))
            if rc != 0:
                raise ValueError("block starts must rise from 0 to n")
        return self

    def __exit__(self, *exc):
        if self.starts is not None:
            lib().orc_set_blocks(0, None)
        return False


class Matrix:
    """Keeps the numpy arrays alive while the C struct points at them."""

    def __init__(self, A):
        self.rowptr = np.ascontiguousarray(A.rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(A.col, dtype=np.int32)
        self.val = np.ascontiguousarray(A.val, dtype=np.float64)
        self.n = int(A.n)
        self.s = OrcMat(self.n, int(self.col.shape[0]), int(getattr(A, "istart", 1)),
                        _ptr(self.rowptr), _ptr(self.col), _ptr(self.val))


def params(solver=1, ipreflag=0, ILU_method=1, precon_thblock=-1, itrmax=1000, rtolmax=1e-8,
           GMRES_m=30, GMRES_GSflag=1, sstep=4, tstep=1, basis=0, qrflag=3) -> OrcParams:
    return OrcParams(solver, ipreflag, ILU_method, precon_thblock, itrmax, rtolmax,
                     GMRES_m, GMRES_GSflag, sstep, tstep, basis, qrflag)


def solve(A, b, x0=None, blocks=None, **kw):
    """Runs the oracle solve; returns (x, reshistory[:niter], niter, iret).  blocks:
    explicit block-Jacobi row starts (see _Blocks)."""
    M = A if isinstance(A, Matrix) else Matrix(A)
    p = params(**kw)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(M.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    hist = np.zeros(max(p.itrmax, 1) + 1)
    niter, iret = C.c_int(0), C.c_int(0)
    with _Blocks(blocks):
        rc = lib().orc_solve(C.byref(M.s), C.byref(p), _ptr(b), _ptr(x), _ptr(hist),
                             C.byref(niter), C.byref(iret))
    if rc != 0:
        return x, hist[:0], 0, rc
    return x, hist[:niter.value].copy(), niter.value, iret.value


def ddcg(A, b_hi, b_lo=None, x0_hi=None, x0_lo=None, a_lo=None, prec_A=2, prec_b=2, prec_x=2, prec_M=2,
         solver=1, blocks=None, **kw):
    """Double-double PCG (ddKSP_pCG, solver=1), BiCGStab (ddKSP_pBiCG, solver=2) or GMRES(m)
    (ddKSP_pGMRES, solver=3, GMRES_m / GMRES_GSflag as for gmres); returns
    (x_hi, x_lo, reshistory[:niter], niter, iret)."""
    M = A if isinstance(A, Matrix) else Matrix(A)
    p = params(solver=solver, **kw)
    f = lambda v: None if v is None else np.ascontiguousarray(v, dtype=np.float64)
    bh, bl, alo = f(b_hi), f(b_lo), f(a_lo)
    xh = np.zeros(M.n) if x0_hi is None else np.array(x0_hi, dtype=np.float64, copy=True)
    xl = np.zeros(M.n) if x0_lo is None else np.array(x0_lo, dtype=np.float64, copy=True)
    hist = np.zeros(max(p.itrmax, 1) + 1)
    niter, iret = C.c_int(0), C.c_int(0)
    ptr = lambda v: None if v is None else _ptr(v)
    with _Blocks(blocks):
        rc = lib().orc_ddcg(C.byref(M.s), ptr(alo), C.byref(p), prec_A, prec_b, prec_x, prec_M, _ptr(bh),
                            ptr(bl), _ptr(xh), _ptr(xl), _ptr(hist), C.byref(niter), C.byref(iret))
    if rc != 0:
        return xh, xl, hist[:0], 0, rc
    return xh, xl, hist[:niter.value].copy(), niter.value, iret.value


def spmv(A, x):
    M = A if isinstance(A, Matrix) else Matrix(A)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty(M.n)
    lib().orc_spmv(C.byref(M.s), _ptr(x), _ptr(y))
    return y


def precon_apply(A, r, blocks=None, **kw):
    M = A if isinstance(A, Matrix) else Matrix(A)
    p = params(**kw)
    r = np.ascontiguousarray(r, dtype=np.float64)
    s = np.zeros(M.n)
    with _Blocks(blocks):
        rc = lib().orc_precon_apply(C.byref(M.s), C.byref(p), _ptr(r), _ptr(s))
    if rc != 0:
        raise RuntimeError(f"oracle preconditioner setup failed: {rc}")
    return s


def true_relres(A, b, x) -> float:
    M = A if isinstance(A, Matrix) else Matrix(A)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().orc_true_relres(C.byref(M.s), _ptr(b), _ptr(x))


def set_threads(t: int) -> None:
    lib().orc_set_threads(int(t))


def num_threads() -> int:
    return lib().orc_num_threads()


class Precon:
    """Persistent oracle preconditioner (setup once, apply many times)."""

    def __init__(self, M: "Matrix", blocks=None, **kw):
        self.M = M
        self.p = params(**kw)
        err = C.c_int(0)
        with _Blocks(blocks):
            self.h = lib().orc_precon_create(C.byref(M.s), C.byref(self.p), C.byref(err))
        if not self.h:
            raise RuntimeError(f"oracle preconditioner setup failed: {err.value}")

    def __call__(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        s = np.empty_like(r)
        lib().orc_precon_apply_h(self.h, _ptr(r), _ptr(s))
        return s

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_precon_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------------------
# DIA format (one process, istart = 1).

class _Crs:
    """Minimal CRS container (1-based rowptr / col) for the oracle's entry points."""

    def __init__(self, n, rowptr, col, val):
        self.n, self.rowptr, self.col, self.val, self.istart = n, rowptr, col, val, 1

    @property
    def nnz(self):
        return int(self.col.shape[0])


def crs_to_dia(A, val=None):
    """get_nnd_crs_without_sort + crs2dia_without_sort (src/matrix.f90:7147-7211, 7494-7534):
    the distinct offsets col - row in ascending order and dia[j*n + k] = A(k, k + offset[j]),
    zero where A has no entry.  val replaces A.val (e.g. the low parts of a dd matrix)."""
    n = int(A.n)
    rp = np.asarray(A.rowptr, dtype=np.int64) - 1
    col = np.asarray(A.col, dtype=np.int64) - 1
    v = np.asarray(A.val if val is None else val, dtype=np.float64)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    d = col - rows
    offsets = np.unique(d)
    j = np.searchsorted(offsets, d)
    dia = np.zeros(len(offsets) * n)
    dia[j * n + rows] = v
    return dia, offsets.astype(np.int32)


def dia_to_crs(dia, offset, n, dia_lo=None):
    """dia2crs (src/matrix.f90:7536-7576) on one process: row k keeps the entries with
    |a| > minReal8 = 0 (src/type.f90:445), here with the diagonals in ascending offset order
    so that the columns are sorted; an entry whose column falls outside rows 1..n (a halo
    column in the reference, zero on one process) is left out.  Returns (CRS, low parts or
    None)."""
    dia = np.asarray(dia, dtype=np.float64).reshape(len(offset), n)
    lo = None if dia_lo is None else np.asarray(dia_lo, dtype=np.float64).reshape(len(offset), n)
    order = np.argsort(np.asarray(offset), kind="stable")
    cols, vals, los, rows = [], [], [], []
    k = np.arange(n, dtype=np.int64)
    for j in order:
        c = k + int(offset[j])
        keep = (c >= 0) & (c < n) & ((np.abs(dia[j]) > 0.0) | ((np.abs(lo[j]) > 0.0) if lo is not None else False))
        rows.append(k[keep]); cols.append(c[keep]); vals.append(dia[j][keep])
        if lo is not None:
            los.append(lo[j][keep])
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    perm = np.lexsort((cols, rows))
    rowptr = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32) + 1
    A = _Crs(n, rowptr, (cols[perm] + 1).astype(np.int32), vals[perm])
    return A, (np.concatenate(los)[perm] if lo is not None else None)


def solve_dia(dia, offset, b, x0=None, **kw):
    """PARCEL_KSP_DIA: the DIA matrix as dia2crs defines it, solved by the CRS oracle."""
    A, _ = dia_to_crs(dia, offset, len(b))
    return solve(A, b, x0, **kw)
