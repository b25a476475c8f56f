"""Python mirror of PARCEL's solver interface on top of libparcelb.

The functions keep the reference's names and argument meaning:

* ``parcel_dcg``, ``parcel_dbicgstab``, ``parcel_dgmres``, ``parcel_dcagmres`` follow the
  Fortran wrappers of src/wrapper.f90 (CPU build 1813-2900, GPU build 362-1455) and their C
  forms in src/example/c2fortran_kernel.f90: CRS 1-based with global column ids, ``vecx``
  holds x0 on entry and the solution on exit, ``reshistory`` (length ``itrmax``) receives
  the relative residual history, and the call returns ``(niter, iret)`` with iret 0 =
  converged, 1 = iteration limit (src/define.f90:101-102) or a negative error code where
  the reference would stop.  Arrays may be numpy (host memory: the C-ABI copies them to
  the GPU and back) or CUDA torch tensors (device memory).
* ``solve`` is PARCEL_KSP_CRS (src/wrapper.f90:47-222) with keyword options named after
  the fields of KSP_INPUT_PARAM.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Crs, load, new_input


def _ptr(a) -> int:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


def _check_types(vecx, vecb, crsA, crsRow_ptr, crsCol):
    for name, a, dt in (("vecx", vecx, "float64"), ("vecb", vecb, "float64"), ("crsA", crsA, "float64"),
                        ("crsRow_ptr", crsRow_ptr, "int32"), ("crsCol", crsCol, "int32")):
        got = str(a.dtype).replace("torch.", "")
        if got != dt:
            raise TypeError(f"{name} must be {dt}, got {got}")


def _i(v):
    return C.byref(C.c_int(int(v)))


def _call_shim(fn, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method,
               addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, Neuman_itr,
               independ_nvec, nBlock, extra=()):
    _check_types(vecx, vecb, crsA, crsRow_ptr, crsCol)
    niter = C.c_int(int(itrmax))
    iret = C.c_int(0)
    hist = reshistory if reshistory is not None else np.zeros(int(itrmax))
    args = [_i(0), _ptr(vecx), _ptr(vecb), C.byref(C.c_int32(n)), C.byref(C.c_int32(gn)),
            C.byref(C.c_int32(nnz)), C.byref(C.c_int32(istart)), _ptr(crsA), _ptr(crsRow_ptr),
            _ptr(crsCol), _i(ipreflag), _i(ILU_method), _i(addL), _i(iflagAS), C.byref(niter),
            C.byref(C.c_double(rtolmax)), _ptr(hist), _i(iovlflag), _i(precon_thblock),
            _i(Neuman_itr), _i(independ_nvec), _i(nBlock)]
    args += [_i(e) for e in extra]
    args += [C.byref(iret)]
    fn(*args)
    return niter.value, iret.value


def _shim_name(base: str, vecx) -> str:
    return base + ("_gpu_c_" if hasattr(vecx, "is_cuda") and vecx.is_cuda else "_c_")


def _dispatch(base, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method,
              addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, Neuman_itr,
              independ_nvec, nBlock, extra=()):
    L = load()
    if hasattr(vecx, "is_cuda") and vecx.is_cuda:
        _check_types(vecx, vecb, crsA, crsRow_ptr, crsCol)
        fn = getattr(L, base + "_gpu_c_")
        niter = C.c_int(int(itrmax))
        iret = C.c_int(0)
        hist = reshistory if reshistory is not None else np.zeros(int(itrmax))
        keep = [C.c_void_p(_ptr(a)) for a in (vecx, vecb, crsA, crsRow_ptr, crsCol)]
        vx, vb, va, vr, vc = (C.byref(k) for k in keep)
        args = [_i(0), vx, vb, C.byref(C.c_int32(n)), C.byref(C.c_int32(gn)), C.byref(C.c_int32(nnz)),
                C.byref(C.c_int32(istart)), va, vr, vc, _i(ipreflag), _i(ILU_method), _i(addL),
                _i(iflagAS), C.byref(niter), C.byref(C.c_double(rtolmax)), _ptr(hist), _i(iovlflag),
                _i(precon_thblock), _i(Neuman_itr), _i(independ_nvec), _i(nBlock)]
        args += [_i(e) for e in extra] + [C.byref(iret)]
        fn(*args)
        return niter.value, iret.value
    return _call_shim(getattr(L, base + "_c_"), vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr,
                      crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory,
                      iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, extra)


def parcel_dcg(vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method, addL,
               iflagAS, itrmax, rtolmax, reshistory, iovlflag=0, precon_thblock=-1, Neuman_itr=1,
               independ_nvec=-1, nBlock=2000):
    """PCG (parcel_dcg, src/wrapper.f90:1995 / :544).  Returns (niter, iret)."""
    return _dispatch("parcel_dcg", vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag,
                     ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock,
                     Neuman_itr, independ_nvec, nBlock)


def parcel_dbicgstab(vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method,
                     addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag=0, precon_thblock=-1,
                     Neuman_itr=1, independ_nvec=-1, nBlock=2000):
    """BiCGStab (parcel_dbicgstab, src/wrapper.f90:1813 / :362).  Returns (niter, iret)."""
    return _dispatch("parcel_dbicgstab", vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol,
                     ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag,
                     precon_thblock, Neuman_itr, independ_nvec, nBlock)


def parcel_dgmres(vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method, addL,
                  iflagAS, itrmax, rtolmax, reshistory, iovlflag=0, precon_thblock=-1, Neuman_itr=1,
                  independ_nvec=-1, nBlock=2000, GMRES_m=4, GMRES_GSflag=1):
    """GMRES(m) (parcel_dgmres, src/wrapper.f90:2179 / :727).  Returns (niter, iret)."""
    return _dispatch("parcel_dgmres", vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag,
                     ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock,
                     Neuman_itr, independ_nvec, nBlock, extra=(GMRES_m, GMRES_GSflag))


def parcel_dcagmres(vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method,
                    addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag=0, precon_thblock=-1,
                    Neuman_itr=1, independ_nvec=-1, nBlock=2000, CAGMRES_sstep=4, CAGMRES_tstep=1,
                    CAGMRES_basis=0, CAGMRES_QRflag=4):
    """CA-GMRES(s,t) (parcel_dcagmres, src/wrapper.f90:2807 / :1355).  Returns (niter, iret)."""
    return _dispatch("parcel_dcagmres", vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol,
                     ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag,
                     precon_thblock, Neuman_itr, independ_nvec, nBlock,
                     extra=(CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag))


def crs_struct(A, rowptr=None, col=None, val=None) -> Crs:
    """parcel_b_crs for a problems.CRS (host) or explicit (device) arrays."""
    rowptr = A.rowptr if rowptr is None else rowptr
    col = A.col if col is None else col
    val = A.val if val is None else val
    return Crs(int(A.n), int(A.n), int(col.shape[0]), int(getattr(A, "istart", 1)), _ptr(rowptr),
               _ptr(col), _ptr(val))


def solve(A, b, x0=None, *, rowptr=None, col=None, val=None, **options):
    """PARCEL_KSP_CRS: solves A x = b with the options of KSP_INPUT_PARAM given as keywords
    (solver, ipreflag, ILU_method, precon_thblock, itrmax, rtolmax, GMRES_m, GMRES_GSflag,
    CAGMRES_*, inner_precision, residual_dd, inner_rtol, max_refine).  Returns a dict with
    x, reshistory, niter, iret and the library's statistics.  Raises on a negative iret."""
    L = load()
    p = new_input(**options)
    S = crs_struct(A, rowptr, col, val)
    on_dev = hasattr(b, "is_cuda") and b.is_cuda
    if x0 is None:
        if on_dev:
            import torch
            x = torch.zeros_like(b)
        else:
            x = np.zeros(A.n)
    else:
        x = x0.clone() if on_dev else np.array(x0, dtype=np.float64, copy=True)
    itrmax = p.itrmax if p.itrmax > 0 else 100
    hist = np.zeros(itrmax)
    niter, iret = C.c_int(0), C.c_int(0)
    rc = L.parcel_b_solve(C.byref(p), C.byref(S), _ptr(b), _ptr(x), _ptr(hist), C.byref(niter),
                          C.byref(iret))
    if rc < 0:
        raise RuntimeError(f"parcel_b_solve failed: {_lib.last_error()}")
    return {"x": x, "reshistory": hist[: niter.value].copy(), "niter": niter.value, "iret": iret.value,
            "stats": _lib.last_stats()}


def ddbicgstab(A, b_hi, b_lo=None, x0_hi=None, x0_lo=None, **kw):
    """The double-double BiCGStab (ddKSP_pBiCG); arguments and result as ddcg."""
    return ddcg(A, b_hi, b_lo, x0_hi, x0_lo, solver=2, **kw)


def ddgmres(A, b_hi, b_lo=None, x0_hi=None, x0_lo=None, **kw):
    """The double-double GMRES(m) (ddKSP_pGMRES; GMRES_m and GMRES_GSflag as for solve);
    arguments and result as ddcg."""
    return ddcg(A, b_hi, b_lo, x0_hi, x0_lo, solver=3, **kw)


def ddcg(A, b_hi, b_lo=None, x0_hi=None, x0_lo=None, *, val_lo=None, rowptr=None, col=None, val=None,
         precision_A=2, precision_b=2, precision_x=2, precision_precondition=2, solver=1, **options):
    """PARCEL_ddKSP_CRS: the double-double PCG (solver=1), BiCGStab (solver=2) or GMRES(m)
    (solver=3) on the GPU.
    Vectors and the matrix's low parts as numpy arrays (host) or CUDA tensors (device).
    Returns a dict with x_hi, x_lo, reshistory, niter, iret and the library's statistics."""
    nnz = int((col if col is not None else A.col).shape[0])
    _check("b_hi", b_hi, "float64", A.n)
    _check("b_lo", b_lo, "float64", A.n)
    _check("x0_hi", x0_hi, "float64", A.n)
    _check("x0_lo", x0_lo, "float64", A.n)
    _check("val_lo", val_lo, "float64", nnz)
    L = load()
    fn = {2: L.parcel_b_ddbicgstab, 3: L.parcel_b_ddgmres}.get(solver, L.parcel_b_ddcg)
    p = new_input(**options)
    S = crs_struct(A, rowptr, col, val)
    on_dev = hasattr(b_hi, "is_cuda") and b_hi.is_cuda

    def fresh(v):
        if v is not None:
            return v.clone() if on_dev else np.array(v, dtype=np.float64, copy=True)
        if on_dev:
            import torch
            return torch.zeros_like(b_hi)
        return np.zeros(A.n)

    xh, xl = fresh(x0_hi), fresh(x0_lo)
    itrmax = p.itrmax if p.itrmax > 0 else 100
    hist = np.zeros(itrmax)
    niter, iret = C.c_int(0), C.c_int(0)
    opt = lambda v: None if v is None else _ptr(v)
    rc = fn(C.byref(p), C.byref(S), opt(val_lo), precision_A, precision_b, precision_x, precision_precondition,
            _ptr(b_hi), opt(b_lo), _ptr(xh), _ptr(xl), _ptr(hist), C.byref(niter), C.byref(iret))
    if rc < 0:
        raise RuntimeError(f"dd solve failed: {_lib.last_error()}")
    return {"x_hi": xh, "x_lo": xl, "reshistory": hist[: niter.value].copy(), "niter": niter.value,
            "iret": iret.value, "stats": _lib.last_stats()}


def _check(name, a, dtype, length=None):
    """Raises before the library is called when an array has the wrong element type or
    length (a wrong type would be read as another type by the C side)."""
    if a is None:
        return
    got = str(a.dtype).replace("torch.", "")
    if got != dtype:
        raise TypeError(f"{name} must be {dtype}, got {got}")
    if length is not None and int(a.shape[0]) != int(length):
        raise ValueError(f"{name} has {int(a.shape[0])} entries, expected {int(length)}")
    dense = a.is_contiguous() if hasattr(a, "is_contiguous") else bool(a.flags.c_contiguous)
    if not dense:
        raise ValueError(f"{name} must be contiguous (the library reads it as a dense array)")


def dia_struct(val, offset, n):
    """parcel_b_dia over DIA arrays (numpy or CUDA tensors): val[j*n + k] is row k's entry on
    the diagonal with column offset offset[j]."""
    return _lib.Dia(int(n), int(n), 1, int(len(offset)), _ptr(val), _ptr(offset))


def solve_dia(val, offset, b, x0=None, **options):
    """PARCEL_KSP_DIA: as solve, for a matrix in DIA format (val: nnd*n doubles, diagonal
    after diagonal; offset: nnd int32 column offsets)."""
    n = int(b.shape[0])
    _check("offset", offset, "int32")
    _check("val", val, "float64", len(offset) * n)
    _check("b", b, "float64")
    _check("x0", x0, "float64", n)
    L = load()
    p = new_input(**options)
    D = dia_struct(val, offset, n)
    on_dev = hasattr(b, "is_cuda") and b.is_cuda
    if x0 is None:
        if on_dev:
            import torch
            x = torch.zeros_like(b)
        else:
            x = np.zeros(n)
    else:
        x = x0.clone() if on_dev else np.array(x0, dtype=np.float64, copy=True)
    itrmax = p.itrmax if p.itrmax > 0 else 100
    hist = np.zeros(itrmax)
    niter, iret = C.c_int(0), C.c_int(0)
    rc = L.parcel_b_solve_dia(C.byref(p), C.byref(D), _ptr(b), _ptr(x), _ptr(hist), C.byref(niter), C.byref(iret))
    if rc < 0:
        raise RuntimeError(f"parcel_b_solve_dia failed: {_lib.last_error()}")
    return {"x": x, "reshistory": hist[: niter.value].copy(), "niter": niter.value, "iret": iret.value,
            "stats": _lib.last_stats()}


def ddsolve_dia(val, offset, b_hi, b_lo=None, x0_hi=None, x0_lo=None, *, val_lo=None, precision_A=2,
                precision_b=2, precision_x=2, precision_precondition=2, solver=1, **options):
    """PARCEL_ddKSP_DIA: the double-double CG (solver=1), BiCGStab (2) or GMRES (3) for a
    matrix in DIA format; arguments and result as ddcg."""
    n = int(b_hi.shape[0])
    _check("offset", offset, "int32")
    _check("val", val, "float64", len(offset) * n)
    _check("val_lo", val_lo, "float64", len(offset) * n)
    _check("b_hi", b_hi, "float64")
    _check("b_lo", b_lo, "float64", n)
    _check("x0_hi", x0_hi, "float64", n)
    _check("x0_lo", x0_lo, "float64", n)
    L = load()
    p = new_input(solver=solver, **options)
    D = dia_struct(val, offset, n)
    xh = np.zeros(n) if x0_hi is None else np.array(x0_hi, dtype=np.float64, copy=True)
    xl = np.zeros(n) if x0_lo is None else np.array(x0_lo, dtype=np.float64, copy=True)
    itrmax = p.itrmax if p.itrmax > 0 else 100
    hist = np.zeros(itrmax)
    niter, iret = C.c_int(0), C.c_int(0)
    opt = lambda v: None if v is None else _ptr(v)
    rc = L.parcel_b_ddsolve_dia(C.byref(p), C.byref(D), opt(val_lo), precision_A, precision_b, precision_x,
                                precision_precondition, _ptr(b_hi), opt(b_lo), _ptr(xh), _ptr(xl), _ptr(hist),
                                C.byref(niter), C.byref(iret))
    if rc < 0:
        raise RuntimeError(f"dd DIA solve failed: {_lib.last_error()}")
    return {"x_hi": xh, "x_lo": xl, "reshistory": hist[: niter.value].copy(), "niter": niter.value,
            "iret": iret.value, "stats": _lib.last_stats()}


class Learned:
    """The learned two-level preconditioner stage (no counterpart in the reference): a
    handle on the network and the coarse solve for an nx x ny x nz grid coarsened by
    ``coarsen`` (even for the stage)."""

    def __init__(self, nx, ny, nz, coarsen, seed=0):
        self._L = load()
        h = C.c_void_p()
        if self._L.parcel_b_learned_create(int(nx), int(ny), int(nz), int(coarsen), int(seed), C.byref(h)) != 0:
            raise RuntimeError(f"parcel_b_learned_create failed: {_lib.last_error()}")
        self.handle = h
        self.grid = (int(nx), int(ny), int(nz), int(coarsen))

    @property
    def coarse_cells(self):
        nx, ny, nz, c = self.grid
        return (nx // c) * (ny // c) * (nz // c)

    def set_stage(self, coarse_steps, use_net):
        """Coarse solve of the stage: Jacobi-PCG iterations, network guess on or off."""
        if self._L.parcel_b_learned_set_stage(self.handle, int(coarse_steps), int(bool(use_net))) != 0:
            raise RuntimeError(f"parcel_b_learned_set_stage failed: {_lib.last_error()}")

    def galerkin(self, A):
        """The stage's 27-tap Galerkin operator for A: array [27][Vc] (float64)."""
        ac = np.zeros((27, self.coarse_cells))
        if self._L.parcel_b_learned_galerkin(self.handle, C.byref(crs_struct(A)), ac.ctypes.data) != 0:
            raise RuntimeError(f"parcel_b_learned_galerkin failed: {_lib.last_error()}")
        return ac

    def coarse_solve(self, A, rc, steps, g0=None):
        """`steps` coarse Jacobi-PCG iterations on P^T A P y = rc (float32), from zero or gamma g0."""
        rc = np.ascontiguousarray(rc, np.float32)
        g = None if g0 is None else np.ascontiguousarray(g0, np.float32)
        y = np.zeros(self.coarse_cells, np.float32)
        rcode = self._L.parcel_b_learned_coarse_solve(self.handle, C.byref(crs_struct(A)), rc.ctypes.data,
                                                      None if g is None else g.ctypes.data, int(steps),
                                                      y.ctypes.data)
        if rcode != 0:
            raise RuntimeError(f"parcel_b_learned_coarse_solve failed: {_lib.last_error()}")
        return y

    def restrict(self, v):
        """P^T v (natural layout, computed in FP32)."""
        v = np.ascontiguousarray(v, np.float64)
        out = np.zeros(self.coarse_cells)
        if self._L.parcel_b_learned_transfer(self.handle, 1, v.ctypes.data, out.ctypes.data) != 0:
            raise RuntimeError(f"parcel_b_learned_transfer failed: {_lib.last_error()}")
        return out

    def prolong(self, y):
        """P y (natural layout, computed in FP32)."""
        nx, ny, nz, _ = self.grid
        y = np.ascontiguousarray(y, np.float64)
        out = np.zeros(nx * ny * nz)
        if self._L.parcel_b_learned_transfer(self.handle, 0, y.ctypes.data, out.ctypes.data) != 0:
            raise RuntimeError(f"parcel_b_learned_transfer failed: {_lib.last_error()}")
        return out

    def collect(self, A, b, max_pairs=16, **options):
        """Appends training pairs from the plain GMRES solve of A x = b (options as in solve)."""
        p = new_input(**options)
        S = crs_struct(A)
        n = C.c_int(0)
        if self._L.parcel_b_learned_collect(self.handle, C.byref(p), C.byref(S), _ptr(b), int(max_pairs),
                                            C.byref(n)) != 0:
            raise RuntimeError(f"parcel_b_learned_collect failed: {_lib.last_error()}")
        return n.value

    def num_pairs(self):
        return self._L.parcel_b_learned_num_pairs(self.handle)

    def train(self, steps, batch=4, lr=1e-3, seed=0):
        """Adam on the collected pairs; returns (first loss, last loss)."""
        f, l = C.c_double(), C.c_double()
        if self._L.parcel_b_learned_train(self.handle, int(steps), int(batch), float(lr), int(seed), C.byref(f),
                                          C.byref(l)) != 0:
            raise RuntimeError(f"parcel_b_learned_train failed: {_lib.last_error()}")
        return f.value, l.value

    def params(self):
        flat = np.zeros(self._L.parcel_b_learned_num_params(), np.float32)
        s = C.c_double()
        self._L.parcel_b_learned_get_params(self.handle, flat.ctypes.data, C.byref(s))
        return flat, s.value

    def set_params(self, flat, scale=0.0):
        flat = np.ascontiguousarray(flat, np.float32)
        if self._L.parcel_b_learned_set_params(self.handle, flat.ctypes.data, float(scale)) != 0:
            raise RuntimeError(_lib.last_error())

    def __del__(self):
        try:
            self._L.parcel_b_learned_destroy(self.handle)
        except Exception:
            pass


def solve_learned(A, b, learned, x0=None, **options):
    """Flexible GMRES with the block-Jacobi ILU / Jacobi preconditioner of ``options`` and
    the learned stage ``learned`` (None: the preconditioner alone).  Returns the dict of
    ``solve``; ``stats["fallback"]`` is 1 when the plain PGMRES path finished the solve."""
    L = load()
    p = new_input(**options)
    S = crs_struct(A)
    x = np.zeros(A.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    itrmax = p.itrmax if p.itrmax > 0 else 100
    hist = np.zeros(itrmax)
    niter, iret = C.c_int(0), C.c_int(0)
    h = learned.handle if learned is not None else None
    rc = L.parcel_b_solve_learned(C.byref(p), C.byref(S), h, _ptr(b), _ptr(x), _ptr(hist), C.byref(niter),
                                  C.byref(iret))
    if rc < 0:
        raise RuntimeError(f"parcel_b_solve_learned failed: {_lib.last_error()}")
    return {"x": x, "reshistory": hist[: niter.value].copy(), "niter": niter.value, "iret": iret.value,
            "stats": _lib.last_stats()}
