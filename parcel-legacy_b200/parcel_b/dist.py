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
(src/pbicg.f90:280-698), KSP_pGMRES (src/pgmres.f90:62-525) and KSP_pCAGMRES
(src/pcagmres.f90:1557-2518), including their iteration-count and return-code conventions,
with every reduction replaced by a distributed one (CA-GMRES reduces a block's Gram and
projection matrices in one message).

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
    options: the parcel_b_input fields (solver 1 = CG, 2 = BiCGStab, 3 = GMRES, 4 = CA-GMRES with
    CAGMRES_sstep / tstep / basis / QRflag; ipreflag, ILU_method,
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
    hist = np.zeros(max(itrmax, 1) + 2)
    if solver == 1:
        niter, iret = _pcg(layout, op, b, x, itrmax, rtol, hist)
    elif solver == 2:
        niter, iret = _pbicg(layout, op, b, x, itrmax, rtol, hist)
    elif solver == 4:
        def opt(name, default, lo):
            v = int(options.get(name, -1))
            return v if v >= lo else default
        niter, iret = _pcagmres(layout, op, b, x, itrmax, rtol, hist, opt("CAGMRES_sstep", 4, 1),
                                opt("CAGMRES_tstep", 1, 1), opt("CAGMRES_basis", BASIS_MONOMIAL, 0),
                                opt("CAGMRES_QRflag", QR_CHOLQR, 1))
    elif solver == 3:
        m = int(options.get("GMRES_m", 4))
        m = m if m > 0 else 4
        niter, iret = _pgmres(layout, op, b, x, itrmax, rtol, hist, m, int(options.get("GMRES_GSflag", 1)) != 2)
    else:
        raise ValueError(f"solver {solver}: the distributed path provides CG (1), BiCGStab (2), GMRES (3) and "
                         "CA-GMRES (4)")
    return niter, iret, hist[:niter].copy()


# ---------------------------------------------------------------- CA-GMRES(s, t)
QR_MGS, QR_CGS, QR_TSQR, QR_CHOLQR, QR_CHOLQR2 = 1, 2, 3, 4, 5
BASIS_MONOMIAL, BASIS_NEWTON = 0, 1


def _sum_ranks(lay, loc: torch.Tensor) -> np.ndarray:
    """A small local array summed over the processes, elementwise, in rank order."""
    loc = loc.reshape(-1).to(torch.float64).contiguous()
    parts = [torch.empty_like(loc) for _ in range(lay.world)]
    dist.all_gather(parts, loc, group=lay.group)
    out = np.zeros(loc.numel())
    for t in parts:
        out = out + t.cpu().numpy()
    return out


def _gram(lay, A: torch.Tensor, B: torch.Tensor) -> np.ndarray:
    """A B^T over the global rows (the panels hold one vector per row): the block inner
    products of calc_gemm_dot (src/pcagmres.f90:1052-1080)."""
    return _sum_ranks(lay, A @ B.T).reshape(A.shape[0], B.shape[0])


def _chol_upper(G):
    """Upper Cholesky factor R (G = R^T R), or None when G is not numerically positive definite."""
    try:
        return np.linalg.cholesky(G).T
    except np.linalg.LinAlgError:
        return None


def _trinv_upper(R):
    return np.triu(np.linalg.inv(np.triu(R)))


def _times_rinv(W: torch.Tensor, Rinv) -> torch.Tensor:
    """The panel W R^-1 (calcQ_VRinv_), one vector per row."""
    return torch.from_numpy(np.ascontiguousarray(Rinv.T)).to(W) @ W


def _qr_r(lay, W: torch.Tensor, flag: int):
    """R-only QR of the global panel W (QRDecomposition_, src/QRDecomposition.f90:1331-1552):
    Cholesky QR or Cholesky QR2 from the distributed Gram matrix, falling back to TSQR when it
    is not numerically positive definite; TSQR (also for the MGS / CGS flags, as on one
    process) as the R of every process's local R factors stacked in rank order, the rows
    signed to a positive diagonal (TSQR_Ronly_)."""
    c = W.shape[0]
    if flag in (QR_CHOLQR, QR_CHOLQR2):
        R1 = _chol_upper(_gram(lay, W, W))
        if R1 is not None:
            if flag == QR_CHOLQR:
                return R1
            Q1 = _times_rinv(W, _trinv_upper(R1))
            R2 = _chol_upper(_gram(lay, Q1, Q1))
            if R2 is not None:
                return R2 @ R1
    loc = torch.linalg.qr(W.T, mode="r").R
    Rl = torch.zeros((c, c), dtype=torch.float64, device=W.device)
    Rl[:loc.shape[0]] = loc
    parts = [torch.empty_like(Rl) for _ in range(lay.world)]
    dist.all_gather(parts, Rl.contiguous(), group=lay.group)
    R = np.linalg.qr(np.concatenate([t.cpu().numpy() for t in parts]), mode="r")
    return R * np.where(np.diag(R) < 0.0, -1.0, 1.0)[:, None]


def _newton_basis(s, B1, er, ei):
    """calc_NewtonBasis (src/pcagmres.f90:586-611): the shifts on B1's diagonal; a complex
    pair (real, +-imaginary) as a 2 x 2 real block."""
    i = 1
    while i <= s:
        B1[i - 1, i - 1] = er[i - 1]
        if i < s and ei[i - 1] != 0.0:
            B1[i, i] = er[i - 1]
            B1[i - 1, i] = -ei[i - 1] * ei[i - 1]
            i += 1
        i += 1


def _leja(er, ei):
    """modified_leja_ordering (src/LejaOrdering.f90:100-322): the Ritz values sorted by
    decreasing modulus, then picked one by one (a complex pair together) to maximise the
    product of distances to those already picked, the values rescaled at every step by the
    growth of that product (the capacity estimate C) and scaled back at the end."""
    n = len(er)
    er, ei = [float(v) for v in er], [float(v) for v in ei]
    mod = lambda j: math.sqrt(er[j] ** 2 + ei[j] ** 2)
    for i in range(1, n):                        # stable insertion sort, largest modulus first
        j = i
        while j > 0 and mod(j - 1) < mod(j):
            er[j], er[j - 1], ei[j], ei[j - 1] = er[j - 1], er[j], ei[j - 1], ei[j]
            j -= 1
    mu = [1.0] * n
    ptmp = [1.0] * n
    tr, ti, picked = [0.0] * n, [0.0] * n, [0] * n
    if ei[0] > 0.0:
        tr[0], ti[0], tr[1], ti[1] = er[0], ei[0], er[1], ei[1]
        picked[0], picked[1] = 0, 1
        L = 2
    else:
        tr[0], ti[0], picked[0] = er[0], 0.0, 0
        L = 1
    C = 1.0
    while L < n:
        c_old = C
        for j in range(L - 1):
            ptmp[j + 1] = math.sqrt((tr[L - 1] - tr[j]) ** 2 + (ti[L - 1] - ti[j]) ** 2) ** (mu[picked[j]] / L)
        C = 1.0
        for v in ptmp:
            C = C * v
        f = C / c_old
        for j in range(n):
            er[j], ei[j], tr[j], ti[j] = er[j] / f, ei[j] / f, tr[j] / f, ti[j] / f
        score = [0.0] * n
        for j in range(n):
            if j not in picked[:L]:
                dists = [math.sqrt((er[j] - tr[q]) ** 2 + (ei[j] - ti[q]) ** 2) ** mu[picked[q]] for q in range(L - 1)]
                prod = 1.0
                for v in dists:
                    prod = prod * v
                score[j] = prod
        k = max(range(n), key=lambda j: (abs(score[j]), -j))
        if abs(ei[k]) > 0.0:
            a, z = (k - 1, k) if ei[k] < 0.0 else (k, k + 1)
            tr[L], ti[L], tr[L + 1], ti[L + 1] = er[a], ei[a], er[z], ei[z]
            picked[L], picked[L + 1] = a, z
            L += 2
        else:
            tr[L], ti[L], picked[L] = er[k], 0.0, k
            L += 1
    return np.array([v * C for v in tr]), np.array([v * C for v in ti])


def _hessenberg_update(s, k, B1, H, R1, Rk, BRup, hk_pre):
    """calc_HessenbergMatrix (src/pcagmres.f90:879-1052): block k's columns of H from its R
    factor, the change-of-basis matrix B1 and the projections BRup on the earlier basis.
    Returns the new subdiagonal entry hk."""
    if k == 1:
        H[: s + 1, :s] = (R1 @ B1) @ _trinv_upper(R1[:s, :s])
        return H[s, s - 1]
    s1 = s * (k - 1)
    Rt = np.zeros((s + 1, s + 1))
    Rt[0, :] = BRup[s1, :]
    Rt[1:, 1:] = Rk
    BRu, BR = BRup[:s1, :], BRup[:s1, :s]
    Rinv = _trinv_upper(Rt[:s, :s])
    H[:s1, s1:s1 + s] = (-(H[:s1, :s1] @ BR) + (BRu @ B1)) @ Rinv
    bk = B1[s, s - 1]
    hk = Rt[s, s] / Rt[s - 1, s - 1] * bk
    H[s * k, s * k - 1] = hk
    Hss = (Rt[:s, :s] @ B1[:s, :s]) @ Rinv
    Hss[:, s - 1] = Hss[:, s - 1] + bk / Rt[s - 1, s - 1] * Rt[:s, s]
    e1 = np.zeros((s, s))
    e1[0, :] = BR[s1 - 1, :] * hk_pre
    H[s1:s1 + s, s1:s1 + s] = Hss - e1 @ Rinv
    return hk


def _pcagmres(lay, op, b, x, itrmax, rtol, hist, s, t, basis, qrflag):
    """KSP_pCAGMRES (src/pcagmres.f90:1557-2518): CA-GMRES(s, t), right preconditioned; per
    block s preconditioned products (monomial, or Newton with Leja-ordered Ritz shifts from
    the second block on), a block Gram-Schmidt against the earlier blocks and an R-only QR,
    all inner products of a block in one distributed reduction."""
    n = lay.n
    st = s * t
    xe = torch.zeros(lay.n_ext, dtype=torch.float64, device=b.device)
    q, pv, w, z = (torch.empty_like(b) for _ in range(4))
    B1 = np.zeros((s + 1, s))
    for i in range(s):
        B1[i + 1, i] = 1.0
    er, ei = np.zeros(st), np.zeros(st)
    bnorm = math.sqrt(lay.dot(b, b))
    exit_now, newton_on = False, False
    itr0, itr = 0, 1
    while itr <= itrmax:
        itr0 = itr
        co, si, ze = np.zeros(st + 1), np.zeros(st + 1), np.zeros(st + 1)
        H, Hg = np.zeros((st + 1, st)), np.zeros((st + 1, st))
        hk_pre = 0.0
        xe[:n] = x
        lay.exchange(xe)
        op.spmv(xe, q)
        r = b - q
        rnorm = math.sqrt(lay.dot(r, r))
        if rnorm / bnorm < rtol:
            break
        if itr == 1:
            hist[0] = rnorm / bnorm
        ze[0] = -rnorm
        V = torch.zeros((s + 1, n), dtype=torch.float64, device=b.device)
        Q = torch.zeros((st + 1, n), dtype=torch.float64, device=b.device)
        V[0] = (-1.0 / rnorm) * r
        mm = 0
        R1 = Rk = BRup = None
        for k in range(1, t + 1):
            if basis == BASIS_NEWTON and newton_on:
                _newton_basis(s, B1, er, ei)
            for i in range(1, s + 1):                  # the basis: V_i = (A M^-1 - shift) V_{i-1}
                op.precon(V[i - 1], pv)
                xe[:n] = pv
                lay.exchange(xe)
                op.spmv(xe, w)
                if basis == BASIS_NEWTON and newton_on:     # calc_NewtonBasisVec (pcagmres.f90:1480-1552)
                    if i != 1:
                        w = (-B1[i - 1, i - 1]) * V[i - 1] + (-B1[i - 2, i - 1]) * V[i - 2] + w
                    else:
                        w = (-B1[i - 1, i - 1]) * V[i - 1] + w
                V[i] = w
            if k == 1:
                R1 = _qr_r(lay, V, qrflag)
                Q[: s + 1] = _times_rinv(V, _trinv_upper(R1))
            else:
                s1 = s * (k - 1) + 1
                BRup = _gram(lay, Q[:s1], V)           # block Gram-Schmidt against the earlier Q
                for c in range(1, s + 1):
                    for j in range(s1):
                        V[c] = V[c] - Q[j] * BRup[j, c]
                Rk = _qr_r(lay, V[1:], qrflag)
                Q[s1:s1 + s] = _times_rinv(V[1:], _trinv_upper(Rk))
            hk_pre = _hessenberg_update(s, k, B1, H, R1, Rk, BRup, hk_pre)
            if k != t:
                V = torch.zeros((s + 1, n), dtype=torch.float64, device=b.device)
                V[0] = Q[s * k]
            Hg[:, s * (k - 1):s * k] = H[:, s * (k - 1):s * k]
            for i in range(s * (k - 1) + 1, s * k + 1):
                mm = i
                _givens(st, Hg, i, co, si, ze)
                rnorm = abs(ze[i])
                itr0 = i + itr
                hist[itr0 - 1] = rnorm / bnorm
                if rnorm / bnorm < rtol or i + itr == itrmax:
                    exit_now = True
                    break
            if exit_now:
                break
            if basis == BASIS_NEWTON:
                newton_on = True
                ev = np.linalg.eigvals(H[: s * k, : s * k])
                er[: s * k], ei[: s * k] = _leja(ev.real, ev.imag)
        # update_xVec: y = Hg^-1 ze over the mm columns, x += M^-1 Q y
        y = np.zeros(mm)
        for i in range(mm, 0, -1):
            v = ze[i - 1]
            for j in range(mm, i, -1):
                v = v - Hg[i - 1, j - 1] * y[j - 1]
            d = Hg[i - 1, i - 1]
            y[i - 1] = v / 1.0e-300 if d == 0.0 else v / d
        v0 = torch.from_numpy(y).to(Q) @ Q[:mm]
        op.precon(v0, z)
        x.add_(z)
        if exit_now:
            break
        itr += st
    return min(itrmax, itr0), (1 if itrmax <= itr else 0)


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


def parcel_dcagmres(x, b, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS,
                    itrmax, rtolmax, reshistory, CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag,
                    group=None, **extra):
    """parcel_dcagmres's argument list (src/wrapper.f90:2807) for one process's rows of a
    distributed matrix; returns (niter, iret)."""
    lay = Layout(n, gn, istart, crsRow_ptr, np.asarray(crsCol)[:nnz], group=group)
    niter, iret, h = solve(lay, np.asarray(crsA)[:nnz], b, x, solver=4, ipreflag=ipreflag, ILU_method=ILU_method,
                           addL=addL, iflagAS=iflagAS, itrmax=itrmax, rtolmax=rtolmax, CAGMRES_sstep=CAGMRES_sstep,
                           CAGMRES_tstep=CAGMRES_tstep, CAGMRES_basis=CAGMRES_basis, CAGMRES_QRflag=CAGMRES_QRflag,
                           **extra)
    reshistory[:len(h)] = h
    return niter, iret


# ---------------------------------------------------------------- DIA rows over processes
def dia_rows(n, gn, istart, diaA, offset, nnd):
    """This process's rows of a DIA matrix as CRS with 1-based global columns.

    PARCEL_KSP_DIA's layout (src/wrapper.f90, src/krylov.f90:845-905): diaA(k + (j-1) n) is
    the entry of global row istart + k - 1 in column row + offset(j); the matrix holds the
    entries of magnitude above zero (get_nnz_dia / dia2crs, src/matrix.f90:7536-7607).  Each
    row's columns come out ascending (the diagonals walked in ascending offset order), a
    column owned by another process becomes a halo column, and a column outside 1..gn (which
    no process owns) is left out.  Returns (rowptr 1-based, col, val)."""
    off = np.asarray(_host_array(offset), dtype=np.int64)[:nnd]
    if len(np.unique(off)) != len(off):
        raise ValueError("a DIA offset appears twice")
    D = np.asarray(_host_array(diaA), dtype=np.float64)[: nnd * n].reshape(nnd, n)
    order = np.argsort(off, kind="stable")
    rows = np.arange(n, dtype=np.int64) + int(istart)
    cols = (rows[None, :] + off[order][:, None]).T            # (n, nnd): row k, ascending offset
    vals = D[order].T
    keep = (np.abs(vals) > 0.0) & (cols >= 1) & (cols <= gn)
    rowptr = np.concatenate([[1], 1 + np.cumsum(keep.sum(axis=1))]).astype(np.int32)
    return rowptr, cols[keep].astype(np.int32), vals[keep]


def _host_array(a):
    return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)


def _dia_solve(solver, x, b, n, gn, istart, diaA, offset, nnd, reshistory, group, options):
    """options["backend"], when given, makes the local operator: backend(layout, val,
    options) (the GPU library's by default)."""
    rowptr, col, val = dia_rows(n, gn, istart, diaA, offset, nnd)
    lay = Layout(n, gn, istart, rowptr, col, group=group)
    make = options.pop("backend", None)
    op = make(lay, val, options) if make is not None else None
    niter, iret, h = solve(lay, val, b, x, backend=op, solver=solver, **options)
    reshistory[:len(h)] = h
    return niter, iret


def parcel_dcg_dia(x, b, n, gn, istart, diaA, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax,
                   reshistory, group=None, **extra):
    """parcel_dcg_dia's argument list (src/wrapper.f90:635) for one process's rows of a
    distributed DIA matrix; returns (niter, iret)."""
    return _dia_solve(1, x, b, n, gn, istart, diaA, offset, nnd, reshistory, group,
                      dict(extra, ipreflag=ipreflag, ILU_method=ILU_method, addL=addL, iflagAS=iflagAS,
                           itrmax=itrmax, rtolmax=rtolmax))


def parcel_dbicgstab_dia(x, b, n, gn, istart, diaA, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax,
                         rtolmax, reshistory, group=None, **extra):
    """parcel_dbicgstab_dia's argument list (src/wrapper.f90:454); returns (niter, iret)."""
    return _dia_solve(2, x, b, n, gn, istart, diaA, offset, nnd, reshistory, group,
                      dict(extra, ipreflag=ipreflag, ILU_method=ILU_method, addL=addL, iflagAS=iflagAS,
                           itrmax=itrmax, rtolmax=rtolmax))


def parcel_dgmres_dia(x, b, n, gn, istart, diaA, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax,
                      reshistory, GMRES_m, GMRES_GSflag, group=None, **extra):
    """parcel_dgmres_dia's argument list (src/wrapper.f90:821); returns (niter, iret)."""
    return _dia_solve(3, x, b, n, gn, istart, diaA, offset, nnd, reshistory, group,
                      dict(extra, ipreflag=ipreflag, ILU_method=ILU_method, addL=addL, iflagAS=iflagAS,
                           itrmax=itrmax, rtolmax=rtolmax, GMRES_m=GMRES_m, GMRES_GSflag=GMRES_GSflag))


def parcel_dcagmres_dia(x, b, n, gn, istart, diaA, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax,
                        rtolmax, reshistory, CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag,
                        group=None, **extra):
    """parcel_dcagmres_dia's argument list (src/wrapper.f90:1457); returns (niter, iret)."""
    return _dia_solve(4, x, b, n, gn, istart, diaA, offset, nnd, reshistory, group,
                      dict(extra, ipreflag=ipreflag, ILU_method=ILU_method, addL=addL, iflagAS=iflagAS,
                           itrmax=itrmax, rtolmax=rtolmax, CAGMRES_sstep=CAGMRES_sstep,
                           CAGMRES_tstep=CAGMRES_tstep, CAGMRES_basis=CAGMRES_basis,
                           CAGMRES_QRflag=CAGMRES_QRflag))
