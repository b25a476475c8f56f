"""Row-distributed preconditioned Krylov solves, one process per GPU.

This mirrors the reference's MPI decomposition, which has no counterpart on one process:
  * every process owns the contiguous rows [istart, istart + n) of the global matrix
    (1-based, global column ids), as src/krylov.f90:447-470 splits them;
  * before every product a process receives the halo values it references from the
    processes that own them (src/comm.f90:153-403, 528-597);
  * block-Jacobi blocks stay inside each process (src/matrix.f90:8074-8134), so the
    preconditioner needs no communication; additive Schwarz with overlap (ipreflag 3,
    addL > 0) extends every block into its neighbours and exchanges addL rows with each
    neighbouring process per application (parcel_b/schwarz.py);
  * an inner product is a local partial followed by one all-gather of the partials,
    summed in rank order, so every process takes the same branch and the result does not
    depend on message timing.

The recurrences are those of KSP_pCG (src/pcg.f90:224-892), KSP_pBiCG
(src/pbicg.f90:280-698) and KSP_pGMRES (src/pgmres.f90:62-525), including their
iteration-count and return-code conventions, with every reduction replaced by the
distributed dot.

Local operations (the product with halo values, the preconditioner) come from a backend
with two methods, ``spmv(x_ext, y)`` and ``precon(r, z)``; the default, ``CudaLocal``, is
the GPU library (parcel_b_local_*) on CUDA tensors.  torch.distributed must be
initialised (NCCL for CUDA tensors); halo messages go through one batched send/receive
per product.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch
import torch.distributed as dist

from . import _lib


class Layout:
    """Row ranges of all processes and this process's halo plan.

    n, istart: this process's row count and first global row (1-based); rowptr, col: its
    rows in CRS (1-based row pointer, 1-based global column ids)."""

    def __init__(self, n: int, gn: int, istart: int, rowptr, col, group=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        ranges = [None] * self.world
        dist.all_gather_object(ranges, (int(istart), int(n)), group=group)
        order = sorted(range(self.world), key=lambda q: ranges[q][0])
        pos = 1
        for q in order:
            if ranges[q][0] != pos:
                raise ValueError(f"rows are not split contiguously: process {q} starts at {ranges[q][0]}, "
                                 f"expected {pos}")
            pos += ranges[q][1]
        if pos - 1 != gn:
            raise ValueError(f"the processes own {pos - 1} rows, gn = {gn}")
        self.n, self.gn, self.istart = int(n), int(gn), int(istart)
        col = np.asarray(col, dtype=np.int64)
        lo, hi = self.istart, self.istart + self.n
        ghost = np.unique(col[(col < lo) | (col >= hi)])
        starts = np.array([ranges[q][0] for q in order])
        owner = np.array([order[i] for i in np.searchsorted(starts, ghost, side="right") - 1], dtype=np.int64)
        self.n_ext = self.n + len(ghost)
        # local column ids: owned rows 1..n, halo values n+1..n_ext in ascending global order
        local = np.empty_like(col)
        own = (col >= lo) & (col < hi)
        local[own] = col[own] - lo + 1
        local[~own] = self.n + 1 + np.searchsorted(ghost, col[~own])
        self.local_col = local.astype(np.int32)
        self.global_col = (col + 0).astype(np.int64)   # 1-based global columns, as given
        self.rowptr = np.asarray(rowptr, dtype=np.int32)
        need = {int(q): ghost[owner == q].tolist() for q in np.unique(owner)}
        needs = [None] * self.world
        dist.all_gather_object(needs, need, group=group)
        # what the others need from this process: local row indices (0-based), in their order
        self.send = {p: np.asarray(needs[p][self.rank], dtype=np.int64) - lo
                     for p in range(self.world) if p != self.rank and self.rank in needs[p]}
        # where the halo values from each owner land: [offset, offset + count) after the n owned
        self.recv = {}
        for q in sorted(need):
            first = int(np.searchsorted(ghost, need[q][0]))
            self.recv[q] = (first, len(need[q]))
        self._send_idx = None

    def exchange(self, x_ext: torch.Tensor) -> None:
        """Fills the halo part x_ext[n:] from the owners' x_ext[:n] (one batched exchange)."""
        if self._send_idx is None:
            self._send_idx = {p: torch.from_numpy(i).to(x_ext.device) for p, i in self.send.items()}
        ops, bufs = [], []
        for p, idx in self._send_idx.items():
            buf = x_ext[:self.n].index_select(0, idx)
            bufs.append(buf)
            ops.append(dist.P2POp(dist.isend, buf, p, group=self.group))
        for q, (off, cnt) in self.recv.items():
            ops.append(dist.P2POp(dist.irecv, x_ext[self.n + off:self.n + off + cnt], q, group=self.group))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def dot(self, a: torch.Tensor, b: torch.Tensor) -> float:
        """Global inner product: local partials gathered and summed in rank order."""
        loc = torch.dot(a, b).reshape(1).to(torch.float64)
        parts = [torch.empty_like(loc) for _ in range(self.world)]
        dist.all_gather(parts, loc, group=self.group)
        s = 0.0
        for t in parts:
            s = s + float(t)
        return s


class CudaLocal:
    """The GPU library's local operator (parcel_b_local_*) for this process's rows."""

    def __init__(self, layout: Layout, val, options: dict):
        from .api import new_input
        self._L = _lib.load()
        if not torch.cuda.is_available():
            raise RuntimeError("the distributed solve runs on the GPU library: no CUDA device")
        # blocks: explicit block-Jacobi row starts of this process (a DDM process's boxes)
        starts = options.get("blocks")
        p = new_input(**{k: v for k, v in options.items() if k != "blocks"})
        rp = np.ascontiguousarray(layout.rowptr, np.int32)
        ci = np.ascontiguousarray(layout.local_col, np.int32)
        va = np.ascontiguousarray(val, np.float64)
        S = _lib.Crs()
        S.n, S.gn, S.nnz, S.istart = layout.n, layout.n, int(ci.shape[0]), 1
        S.rowptr, S.col, S.val = rp.ctypes.data, ci.ctypes.data, va.ctypes.data
        h = C.c_void_p()
        if starts is None:
            rc = self._L.parcel_b_local_create(C.byref(p), C.byref(S), layout.n_ext, C.byref(h))
        else:
            st = np.ascontiguousarray(starts, np.int32)
            rc = self._L.parcel_b_local_create_blocks(C.byref(p), C.byref(S), layout.n_ext, len(st) - 1,
                                                      st.ctypes.data_as(_lib.I32P), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"parcel_b_local_create failed: {_lib.last_error()}")
        self.h = h

    def spmv(self, x_ext: torch.Tensor, y: torch.Tensor) -> None:
        if self._L.parcel_b_local_spmv(self.h, x_ext.data_ptr(), y.data_ptr()) != 0:
            raise RuntimeError(f"parcel_b_local_spmv failed: {_lib.last_error()}")

    def precon(self, r: torch.Tensor, z: torch.Tensor) -> None:
        if self._L.parcel_b_local_precon(self.h, r.data_ptr(), z.data_ptr()) != 0:
            raise RuntimeError(f"parcel_b_local_precon failed: {_lib.last_error()}")

    def __del__(self):
        try:
            self._L.parcel_b_local_destroy(self.h)
        except Exception:
            pass


def _pcg(lay, op, b, x, itrmax, rtol, hist):
    """KSP_pCG (src/pcg.f90:224-892): preconditioned CG with the lagged x update."""
    n = lay.n
    xe = torch.zeros(lay.n_ext, dtype=torch.float64, device=b.device)
    r, q, s = torch.empty_like(b), torch.empty_like(b), torch.empty_like(b)
    p = torch.zeros_like(b)
    xe[:n] = x
    lay.exchange(xe)
    op.spmv(xe, q)
    torch.sub(b, q, out=r)
    bnorm = math.sqrt(lay.dot(b, b))
    rnorm = math.sqrt(lay.dot(r, r))
    alpha = beta = 0.0
    op.precon(r, s)
    rho0 = lay.dot(s, r)
    itr = 0
    for itr in range(1, itrmax + 1):
        hist[itr - 1] = rnorm / bnorm
        x.add_(p, alpha=alpha)                 # CG_axpy2 (pcg.f90:4-20)
        p.mul_(beta).add_(s)
        xe[:n] = p
        lay.exchange(xe)
        op.spmv(xe, q)
        gamma = lay.dot(p, q)
        alpha = rho0 / gamma
        r.add_(q, alpha=-alpha)
        op.precon(r, s)
        rho1 = lay.dot(s, r)                    # CG_calc_dot2 (pcg.f90:22-53)
        rnorm = math.sqrt(lay.dot(r, r))
        if rnorm / bnorm < rtol or rnorm / bnorm > 1.0e8:
            break
        beta = rho1 / rho0
        rho0 = rho1
    x.add_(p, alpha=alpha)
    return min(itrmax, itr), (1 if itrmax <= itr else 0)


def _pbicg(lay, op, b, x, itrmax, rtol, hist):
    """KSP_pBiCG (src/pbicg.f90:280-698): right-preconditioned BiCGStab, two products and two
    preconditioner applications per iteration, every inner product a distributed dot."""
    n = lay.n
    xe = torch.zeros(lay.n_ext, dtype=torch.float64, device=b.device)
    r = torch.empty_like(b)
    q, pp, e, pe, v = (torch.zeros_like(b) for _ in range(5))
    xe[:n] = x
    lay.exchange(xe)
    op.spmv(xe, q)
    torch.sub(b, q, out=r)                     # calc_res
    bnorm = math.sqrt(lay.dot(b, b))
    rnorm = math.sqrt(lay.dot(r, r))
    r0, p = r.clone(), r.clone()
    c1 = lay.dot(r0, r0)
    itr = 0
    for itr in range(1, itrmax + 1):
        hist[itr - 1] = rnorm / bnorm
        op.precon(p, pp)                       # pp = M^-1 p
        xe[:n] = pp
        lay.exchange(xe)
        op.spmv(xe, q)                         # q = A pp
        c2 = lay.dot(r0, q)
        alpha = c1 / c2
        torch.add(r, q, alpha=-alpha, out=e)   # e = r - alpha q
        op.precon(e, pe)                       # pe = M^-1 e
        xe[:n] = pe
        lay.exchange(xe)
        op.spmv(xe, v)                         # v = A pe
        c3 = lay.dot(e, v) / lay.dot(v, v)
        x.add_(pp, alpha=alpha).add_(pe, alpha=c3)
        torch.add(e, v, alpha=-c3, out=r)      # r = e - c3 v
        c1 = lay.dot(r, r0)
        rnorm = math.sqrt(lay.dot(r, r))
        if rnorm / bnorm < rtol:
            break
        beta = c1 / (c3 * c2)
        p.mul_(beta).add_(q, alpha=-beta * c3).add_(r)   # p = r - beta c3 q + beta p
    return min(itrmax, itr), (1 if itrmax <= itr else 0)


def _givens(m, h, i, c, s, e):
    """GivensRotations (src/pcagmres.f90:190-242) on column i (1-based) of h[(m+1) x m],
    with the reference's zero-diagonal guard h/1.0d0-300 (Fortran: (h/1) - 300)."""
    col = h[:, i - 1]
    for k in range(1, i):
        t1 = col[k - 1] * c[k - 1] - col[k] * s[k - 1]
        t2 = col[k - 1] * s[k - 1] + col[k] * c[k - 1]
        col[k - 1], col[k] = t1, t2
    t = col[i] / 1.0 - 300.0 if col[i - 1] == 0.0 else col[i] / col[i - 1]
    c[i - 1] = 1.0 / math.sqrt(1.0 + t * t)
    s[i - 1] = -c[i - 1] * t
    t1 = c[i - 1] * e[i - 1] - s[i - 1] * e[i]
    t2 = s[i - 1] * e[i - 1] + c[i - 1] * e[i]
    e[i - 1], e[i] = t1, t2
    col[i - 1] = c[i - 1] * col[i - 1] - s[i - 1] * col[i]
    col[i] = 0.0


def _pgmres(lay, op, b, x, itrmax, rtol, hist, m, mgs):
    """KSP_pGMRES (src/pgmres.f90:62-525): right-preconditioned GMRES(m), MGS or CGS."""
    n = lay.n
    dev = b.device
    V = torch.zeros((m + 1, n), dtype=torch.float64, device=dev)
    xe = torch.zeros(lay.n_ext, dtype=torch.float64, device=dev)
    r, w, pv = torch.empty_like(b), torch.empty_like(b), torch.empty_like(b)
    bnorm = math.sqrt(lay.dot(b, b))
    rnorm = 0.0
    itr, inner, mm = 1, 1, 0
    while itr <= itrmax:
        h = np.zeros((m + 1, m))
        c, s, e = np.zeros(m + 1), np.zeros(m + 1), np.zeros(m + 1)
        xe[:n] = x
        lay.exchange(xe)
        op.spmv(xe, r)
        torch.sub(b, r, out=r)
        rnorm = math.sqrt(lay.dot(r, r))
        torch.mul(r, -1.0 / rnorm, out=V[0])
        e[0] = -rnorm
        if rnorm / bnorm < rtol:
            break
        if itr == 1:
            hist[0] = rnorm / bnorm
        exit_inner = False
        for inner in range(1, m + 1):
            op.precon(V[inner - 1], pv)
            xe[:n] = pv
            lay.exchange(xe)
            op.spmv(xe, w)
            if mgs:
                for k in range(1, inner + 1):
                    hk = lay.dot(w, V[k - 1])
                    h[k - 1, inner - 1] = hk
                    w.add_(V[k - 1], alpha=-hk)
            else:                               # CGS_Orth (pgmres.f90:11-58)
                hk = [lay.dot(w, V[k - 1]) for k in range(1, inner + 1)]
                for k in range(1, inner + 1):
                    w.add_(V[k - 1], alpha=-hk[k - 1])
                    h[k - 1, inner - 1] = hk[k - 1]
            wn = math.sqrt(lay.dot(w, w))
            h[inner, inner - 1] = wn
            torch.mul(w, 1.0 / wn, out=V[inner])
            _givens(m, h, inner, c, s, e)
            rnorm = abs(e[inner])
            mm = inner
            if itr + inner <= itrmax:
                hist[itr + inner - 1] = rnorm / bnorm
            if rnorm / bnorm < rtol or itr + inner == itrmax:
                exit_inner = True
                break
        if not exit_inner:
            inner = m + 1                       # the Fortran DO variable after completion
        mm = min(mm, m)
        # update_xVec (pcagmres.f90:1136-1236): y = H^-1 e, v0 = V y, x += M^-1 v0
        y = np.zeros(m + 1)
        for i in range(mm, 0, -1):
            y[i - 1] = e[i - 1]
            for j in range(mm, i, -1):
                y[i - 1] = y[i - 1] - h[i - 1, j - 1] * y[j - 1]
            d = h[i - 1, i - 1]
            y[i - 1] = y[i - 1] / 1.0e-300 if d == 0.0 else y[i - 1] / d
        v0 = torch.zeros_like(b)
        for i in range(mm):
            v0.add_(V[i], alpha=float(y[i]))
        op.precon(v0, pv)
        x.add_(pv)
        if rnorm / bnorm < rtol or itr + inner == itrmax:
            break
        itr += m
    return min(itrmax, itr + inner), (1 if itrmax <= itr else 0)


def cuda_block_precon(n, rowptr, col, val, starts, options):
    """The library's block-Jacobi operator of an n-row matrix without halo columns (1-based
    local rowptr / col), with explicit blocks `starts`: precon(r, z) on CUDA tensors."""
    import types
    lay = types.SimpleNamespace(n=int(n), n_ext=int(n), rowptr=np.asarray(rowptr, np.int32),
                                local_col=np.asarray(col, np.int32))
    return CudaLocal(lay, val, dict(options, blocks=starts))


class _Composed:
    """The product of one local operator and the preconditioner of another."""

    def __init__(self, spmv_op, precon_op):
        self.s, self.p = spmv_op, precon_op

    def spmv(self, x_ext, y):
        self.s.spmv(x_ext, y)

    def precon(self, r, z):
        self.p.precon(r, z)


def solve(layout: Layout, val, b: torch.Tensor, x: torch.Tensor, backend=None, **options):
    """Distributed solve of the rows this process owns.  b, x: this process's parts
    (float64 tensors on the backend's device; x is the initial guess and the result).
    options: the parcel_b_input fields (solver 1 = CG, 2 = BiCGStab, 3 = GMRES; ipreflag, ILU_method,
    precon_thblock = block-Jacobi blocks of this process, itrmax, rtolmax, GMRES_m,
    GMRES_GSflag) and, for the default backend, blocks = explicit block-Jacobi row starts of
    this process.  Returns (niter, iret, reshistory)."""
    solver = int(options.get("solver", 3))
    itrmax = int(options.get("itrmax", 100))
    rtol = float(options.get("rtolmax", 1e-8))
    if backend is not None:
        op = backend
    elif int(options.get("ipreflag", 0)) == 3 and layout.world > 1:
        # additive Schwarz with overlap (parcel_b/schwarz.py): the product from a local operator
        # without preconditioner, the preconditioner from the overlapped regions
        from .schwarz import Schwarz
        base = CudaLocal(layout, val, dict(options, ipreflag=0))
        ilu = int(options.get("ILU_method", 1))
        prec = Schwarz(layout, layout.rowptr, layout.global_col, val, int(options.get("precon_thblock", 1)),
                       int(options.get("addL", 0)), int(options.get("iflagAS", 1)), ilu if ilu > 0 else 1,
                       cuda_block_precon, {k: v for k, v in options.items() if k not in ("addL", "iflagAS")})
        op = _Composed(base, prec)
    else:
        op = CudaLocal(layout, val, options)
    hist = np.zeros(max(itrmax, 1))
    if solver == 1:
        niter, iret = _pcg(layout, op, b, x, itrmax, rtol, hist)
    elif solver == 2:
        niter, iret = _pbicg(layout, op, b, x, itrmax, rtol, hist)
    elif solver == 3:
        m = int(options.get("GMRES_m", 4))
        m = m if m > 0 else 4
        niter, iret = _pgmres(layout, op, b, x, itrmax, rtol, hist, m, int(options.get("GMRES_GSflag", 1)) != 2)
    else:
        raise ValueError(f"solver {solver}: the distributed path provides CG (1), BiCGStab (2) and GMRES (3)")
    return niter, iret, hist[:niter].copy()


def parcel_dcg(x, b, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax,
               rtolmax, reshistory, group=None, **extra):
    """parcel_dcg's argument list (src/wrapper.f90:1995) for one process's rows of a
    distributed matrix; returns (niter, iret)."""
    lay = Layout(n, gn, istart, crsRow_ptr, np.asarray(crsCol)[:nnz], group=group)
    niter, iret, h = solve(lay, np.asarray(crsA)[:nnz], b, x, solver=1, ipreflag=ipreflag, ILU_method=ILU_method,
                           addL=addL, iflagAS=iflagAS,
                           itrmax=itrmax, rtolmax=rtolmax, **extra)
    reshistory[:len(h)] = h
    return niter, iret


def parcel_dbicgstab(x, b, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS,
                     itrmax, rtolmax, reshistory, group=None, **extra):
    """parcel_dbicgstab's argument list (src/wrapper.f90:1813) for one process's rows of a
    distributed matrix; returns (niter, iret)."""
    lay = Layout(n, gn, istart, crsRow_ptr, np.asarray(crsCol)[:nnz], group=group)
    niter, iret, h = solve(lay, np.asarray(crsA)[:nnz], b, x, solver=2, ipreflag=ipreflag, ILU_method=ILU_method,
                           addL=addL, iflagAS=iflagAS,
                           itrmax=itrmax, rtolmax=rtolmax, **extra)
    reshistory[:len(h)] = h
    return niter, iret


def parcel_dgmres(x, b, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax,
                  rtolmax, reshistory, GMRES_m, GMRES_GSflag, group=None, **extra):
    """parcel_dgmres's argument list (src/wrapper.f90:2179) for one process's rows of a
    distributed matrix; returns (niter, iret)."""
    lay = Layout(n, gn, istart, crsRow_ptr, np.asarray(crsCol)[:nnz], group=group)
    niter, iret, h = solve(lay, np.asarray(crsA)[:nnz], b, x, solver=3, ipreflag=ipreflag, ILU_method=ILU_method,
                           addL=addL, iflagAS=iflagAS,
                           itrmax=itrmax, rtolmax=rtolmax, GMRES_m=GMRES_m, GMRES_GSflag=GMRES_GSflag, **extra)
    reshistory[:len(h)] = h
    return niter, iret
