"""DDM stencil-format solves (src/src_DDM): each process holds its box of a structured grid.

A DDM matrix is one process's box, padded by `margin` cells on both sides of every axis,
x fastest: m = prod(n_d + 2 margin) cells; stencil point k couples interior cell j with
cell j + offset[k] with the value val[k m + j] (set_grids_decompostion and
make_poisson_3D_DDM, src/example/ddm_setup.f90).  b and x hold m entries; the interior
cells carry the unknowns.

* ``solve`` / ``ddsolve``: one process's whole grid through parcel_b_solve_ddm /
  parcel_b_ddsolve_ddm (the GPU library), numpy arrays or CUDA tensors.
* ``parcel_dcg_ddm`` / ``parcel_dbicgstab_ddm`` / ``parcel_dgmres_ddm`` /
  ``parcel_dcagmres_ddm``: the argument lists of the reference's functions of those names
  (src/src_DDM/ddm_kernel.f90:2893-2986, 2988-3080, 3082-3178, 3180-3279) for a
  box that is one of several processes' (torch.distributed, one process per GPU, ranks laid
  out as set_rank_xyz lays them out, src/example/ddm_setup.f90:52-60).  Every process
  numbers its interior cells box by box after the lower ranks' cells; a margin cell it
  couples to is a neighbour's interior cell, whose value arrives before every product
  through parcel_b.dist's halo exchange (the reference's sleeve exchange); the block-Jacobi
  boxes stay inside the process, as the reference's per-process D-ILU does.  With one
  process these are ``solve``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import load, new_input
from .api import _check, _ptr

BOXES_THREADS = 0   # CPU build: precon_thblock slabs along div_direc_th
BOXES_CUBES = 1     # CUDA build (DDM_CUDA_BJ): n_d / 4 boxes per axis


def ddm_struct(val, offset, offset_dim, n_grids, margin=1, div_direc_th=1, boxes=BOXES_THREADS):
    """parcel_b_ddm over the arrays (numpy or CUDA tensors; offset_dim as the reference's
    offset_dim(nnd, ndim), column-major)."""
    ndim = len(n_grids)
    pad = [int(v) + 2 * int(margin) for v in n_grids]
    D = _lib.Ddm()
    D.ndim = ndim
    for d in range(ndim):
        D.n_grids[d] = int(n_grids[d])
    D.margin = int(margin)
    D.m = int(np.prod(pad))
    D.nnd = int(len(offset))
    D.offset, D.offset_dim, D.val = _ptr(offset), _ptr(offset_dim), _ptr(val)
    D.div_direc_th = int(div_direc_th)
    D.boxes = int(boxes)
    return D


def order(n_grids, nnd, margin=1, div_direc_th=1, boxes=BOXES_THREADS, precon_thblock=-1):
    """The renumbering the library applies to a box: perm[r] (padded cell of row r) and the
    row starts of the block-Jacobi boxes (parcel_b_ddm_order; host-side, no GPU needed)."""
    D = ddm_struct(None, np.zeros(nnd, np.int32), None, n_grids, margin, div_direc_th, boxes)
    D.offset = None
    L = load()
    nb = C.c_int32(0)
    L.parcel_b_ddm_order(C.byref(D), int(precon_thblock), None, None, C.byref(nb))
    nint = int(np.prod([int(v) for v in n_grids]))
    perm = np.empty(nint, np.int32)
    starts = np.empty(nb.value + 1, np.int32)
    rc = L.parcel_b_ddm_order(C.byref(D), int(precon_thblock), perm.ctypes.data_as(_lib.I32P),
                              starts.ctypes.data_as(_lib.I32P), C.byref(nb))
    if rc < 0:
        raise RuntimeError(f"parcel_b_ddm_order failed: {_lib.last_error()}")
    return perm, starts


def _m_of(n_grids, margin):
    return int(np.prod([int(v) + 2 * int(margin) for v in n_grids]))


def solve(val, offset, offset_dim, n_grids, b, x0=None, *, margin=1, div_direc_th=1, boxes=BOXES_THREADS,
          out=None, **options):
    """parcel_ddm_main on one process: the Krylov solver and preconditioner of the options
    (solver 1-4, ipreflag 0-2, precon_thblock, itrmax, rtolmax, GMRES_m, ...) on the interior
    cells.  Returns {x, reshistory, niter, iret, stats}; x's margin entries are x0's.

    out: an array of m float64 (host, or a device tensor when b is one) that holds the initial
    guess on entry and receives x in place, as the reference's x argument does; x0 must then
    be None.  A caller that keeps out in page-locked memory gets full-speed copies."""
    m = _m_of(n_grids, margin)
    _check("offset", offset, "int32")
    _check("offset_dim", offset_dim, "int32", len(offset) * len(n_grids))
    _check("val", val, "float64", len(offset) * m)
    _check("b", b, "float64", m)
    _check("x0", x0, "float64", m)
    _check("out", out, "float64", m)
    on_dev = hasattr(b, "is_cuda") and b.is_cuda
    if out is not None:
        if x0 is not None:
            raise ValueError("give the initial guess in out, not in x0, when out is given")
        if on_dev != (hasattr(out, "is_cuda") and out.is_cuda):
            raise ValueError("out must be on the device when b is, and on the host when b is")
        x = out
    elif x0 is None:
        if on_dev:
            import torch
            x = torch.zeros_like(b)
        else:
            x = np.zeros(m)
    else:
        x = x0.clone() if on_dev else np.array(x0, dtype=np.float64, copy=True)
    L = load()
    p = new_input(**options)
    D = ddm_struct(val, offset, offset_dim, n_grids, margin, div_direc_th, boxes)
    itrmax = p.itrmax if p.itrmax > 0 else 100
    hist = np.zeros(itrmax)
    niter, iret = C.c_int(0), C.c_int(0)
    rc = L.parcel_b_solve_ddm(C.byref(p), C.byref(D), _ptr(b), _ptr(x), _ptr(hist), C.byref(niter), C.byref(iret))
    if rc < 0:
        raise RuntimeError(f"parcel_b_solve_ddm failed: {_lib.last_error()}")
    return {"x": x, "reshistory": hist[: niter.value].copy(), "niter": niter.value, "iret": iret.value,
            "stats": _lib.last_stats()}


def ddsolve(val, offset, offset_dim, n_grids, b_hi, b_lo=None, x0_hi=None, x0_lo=None, *, val_lo=None, margin=1,
            div_direc_th=1, boxes=BOXES_THREADS, precision_A=2, precision_b=2, precision_x=2,
            precision_precondition=2, solver=1, **options):
    """parcel_ddm_main_dd on one process: the double-double CG (1), BiCGStab (2) or GMRES (3);
    returns {x_hi, x_lo, reshistory, niter, iret, stats}."""
    m = _m_of(n_grids, margin)
    _check("offset", offset, "int32")
    _check("val", val, "float64", len(offset) * m)
    _check("val_lo", val_lo, "float64", len(offset) * m)
    _check("b_hi", b_hi, "float64", m)
    _check("b_lo", b_lo, "float64", m)
    xh = np.zeros(m) if x0_hi is None else np.array(x0_hi, dtype=np.float64, copy=True)
    xl = np.zeros(m) if x0_lo is None else np.array(x0_lo, dtype=np.float64, copy=True)
    L = load()
    p = new_input(solver=solver, **options)
    D = ddm_struct(val, offset, offset_dim, n_grids, margin, div_direc_th, boxes)
    itrmax = p.itrmax if p.itrmax > 0 else 100
    hist = np.zeros(itrmax)
    niter, iret = C.c_int(0), C.c_int(0)
    opt = lambda v: None if v is None else _ptr(v)
    rc = L.parcel_b_ddsolve_ddm(C.byref(p), C.byref(D), opt(val_lo), precision_A, precision_b, precision_x,
                                precision_precondition, _ptr(b_hi), opt(b_lo), _ptr(xh), _ptr(xl), _ptr(hist),
                                C.byref(niter), C.byref(iret))
    if rc < 0:
        raise RuntimeError(f"parcel_b_ddsolve_ddm failed: {_lib.last_error()}")
    return {"x_hi": xh, "x_lo": xl, "reshistory": hist[: niter.value].copy(), "niter": niter.value,
            "iret": iret.value, "stats": _lib.last_stats()}


# ---- several processes --------------------------------------------------------------------
def rank_xyz(rank, npe):
    """set_rank_xyz: rank = npe_x npe_y rz + npe_x ry + rx."""
    px, py = int(npe[0]), int(npe[1]) if len(npe) > 1 else 1
    return (rank % (px * py)) % px, (rank % (px * py)) // px, rank // (px * py)


def _host(a):
    """A host numpy view of an array or tensor."""
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def _dims3(v, fill):
    v = [int(a) for a in v]
    return v + [fill] * (3 - len(v))


class Decomposition:
    """This process's share of a DDM decomposition over torch.distributed: the global
    numbering of its interior cells, the columns of its couplings, the dist.Layout of its rows
    and its block-Jacobi boxes.

    val, offset, offset_dim, n_grids, npe_dim, margin: this process's DDM arguments; boxes,
    div_direc_th, precon_thblock: how its boxes are cut (the same on every process)."""

    def __init__(self, val, offset, offset_dim, n_grids, npe_dim, margin=1, div_direc_th=1, boxes=BOXES_THREADS,
                 precon_thblock=-1, group=None):
        import torch.distributed as dist

        from .dist import Layout
        ndim = len(n_grids)
        nnd = len(offset)
        self.group = group
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        npe = _dims3(npe_dim, 1)
        if int(np.prod(npe)) != world:
            raise ValueError(f"npe_dim {list(npe_dim)} does not match {world} processes")
        me = rank_xyz(rank, npe)
        n = _dims3(n_grids, 1)
        sizes = [None] * world
        dist.all_gather_object(sizes, n, group=group)
        mg = [int(margin)] * ndim + [0] * (3 - ndim)
        pad = [n[d] + 2 * mg[d] for d in range(3)]
        m = int(np.prod(pad))
        stride = [1, pad[0], pad[0] * pad[1]]
        self.n_int = int(np.prod(n))
        nint = [int(np.prod(s)) for s in sizes]
        base = np.concatenate([[0], np.cumsum(nint)]).astype(np.int64)
        self.base, self.gn = int(base[rank]), int(base[-1])
        od = _host(offset_dim).astype(np.int64).reshape(ndim, nnd).T
        od = np.concatenate([od, np.zeros((nnd, 3 - ndim), np.int64)], axis=1)
        off = _host(offset).astype(np.int64)
        if not np.array_equal(off, od @ np.array(stride, np.int64)):
            raise ValueError("offset and offset_dim describe different stencils")
        if np.abs(od).max() > int(margin):
            raise ValueError("a stencil point reaches beyond the margin")

        def coords_rank(c):
            return c[0] + npe[0] * (c[1] + npe[1] * c[2])

        kw = dict(margin=margin, div_direc_th=div_direc_th, boxes=boxes, precon_thblock=precon_thblock)
        self.perm, self.starts = order(n[:ndim], nnd, **kw)
        perm = self.perm.astype(np.int64)
        inv_cache = {}

        def inv_of(q):
            """Row of every padded cell of process q (-1 on the margin)."""
            if q not in inv_cache:
                sq = sizes[q]
                pq = self.perm if q == rank else order(sq[:ndim], nnd, **kw)[0]
                inv = np.full(int(np.prod([sq[d] + 2 * mg[d] for d in range(3)])), -1, np.int64)
                inv[pq.astype(np.int64)] = np.arange(len(pq))
                inv_cache[q] = inv
            return inv_cache[q]

        vals = _host(val).astype(np.float64)
        # interior coordinates of every row
        cx = perm % pad[0] - mg[0]
        cy = (perm // pad[0]) % pad[1] - mg[1]
        cz = perm // (pad[0] * pad[1]) - mg[2]
        rows, cols, vv = [], [], []
        r_all = np.arange(self.n_int, dtype=np.int64)
        for k in range(nnd):
            v = vals[k * m + perm]
            tx, ty, tz = cx + od[k, 0], cy + od[k, 1], cz + od[k, 2]
            # neighbouring process along each axis: -1, 0 or +1
            dx = np.where(tx < 0, -1, np.where(tx >= n[0], 1, 0))
            dy = np.where(ty < 0, -1, np.where(ty >= n[1], 1, 0))
            dz = np.where(tz < 0, -1, np.where(tz >= n[2], 1, 0))
            keep = v != 0.0
            for sx, sy, sz in {(int(a), int(b_), int(c)) for a, b_, c in zip(dx[keep], dy[keep], dz[keep])}:
                sel = keep & (dx == sx) & (dy == sy) & (dz == sz)
                nb = (me[0] + sx, me[1] + sy, me[2] + sz)
                if not all(0 <= nb[d] < npe[d] for d in range(3)):
                    continue   # outside the grid: the margin cell stays zero in the reference
                q = coords_rank(nb)
                sq = sizes[q]
                ux = tx[sel] - (n[0] if sx > 0 else 0) + (sq[0] if sx < 0 else 0)
                uy = ty[sel] - (n[1] if sy > 0 else 0) + (sq[1] if sy < 0 else 0)
                uz = tz[sel] - (n[2] if sz > 0 else 0) + (sq[2] if sz < 0 else 0)
                if (ux < 0).any() or (ux >= sq[0]).any() or (uy < 0).any() or (uy >= sq[1]).any() or \
                        (uz < 0).any() or (uz >= sq[2]).any():
                    raise ValueError("a stencil point reaches past the neighbouring process's box")
                qp = [sq[d] + 2 * mg[d] for d in range(3)]
                pj = (ux + mg[0]) + qp[0] * ((uy + mg[1]) + qp[1] * (uz + mg[2]))
                rows.append(r_all[sel])
                cols.append(base[q] + inv_of(q)[pj])
                vv.append(v[sel])
        rows, cols, vv = np.concatenate(rows), np.concatenate(cols), np.concatenate(vv)
        o = np.lexsort((cols, rows))
        rows, cols, self.val = rows[o], cols[o], vv[o]
        rowptr = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=self.n_int))]) + 1
        self.layout = Layout(self.n_int, self.gn, self.base + 1, rowptr.astype(np.int32), cols + 1, group=group)
        self.m = m

    def _index(self, v):
        import torch
        return torch.from_numpy(self.perm.astype(np.int64)).to(v.device)

    def to_rows(self, v):
        """The interior entries of a padded tensor, in row order."""
        return v[self._index(v)]

    def to_box(self, rows, v):
        """Writes rows back into the padded tensor v (margin untouched)."""
        v[self._index(v)] = rows


def _distributed(solver, x, b, m, nnd, offset, diaA, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th,
                 ipreflag, itrmax, rtolmax, reshistory, precon_thblock, independ_nvec, group, boxes, backend,
                 **extra):
    import torch

    from . import dist as pdist
    if ipreflag not in (0, 1, 2):
        raise ValueError(f"ipreflag = {ipreflag}: the DDM path provides none, point Jacobi and block-Jacobi D-ILU")
    if independ_nvec == 1:
        raise ValueError("independ_nvec = 1 (the x-line-independent DDM D-ILU) is not provided")
    dec = Decomposition(_host(diaA)[:nnd * m], offset, offset_dim, list(n_grids)[:ndim], npe_dim, margin,
                        div_direc_th, boxes, precon_thblock, group)
    xt = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.asarray(x))
    bt = b if isinstance(b, torch.Tensor) else torch.from_numpy(np.asarray(b))
    xr, br = dec.to_rows(xt).clone(), dec.to_rows(bt).clone()
    opts = dict(solver=solver, ipreflag=ipreflag, ILU_method=1, itrmax=itrmax, rtolmax=rtolmax, **extra)
    be = None
    if backend is not None:
        be = backend(dec.layout, dec.val, dec.starts, opts)
    else:
        opts["blocks"] = dec.starts
    niter, iret, h = pdist.solve(dec.layout, dec.val, br, xr, backend=be, **opts)
    dec.to_box(xr, xt)   # xt shares memory with a numpy x
    reshistory[:len(h)] = h
    return niter, iret


def parcel_dcg_ddm(x, b, m, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim, npe_dim, n_grids,
                   offset_dim, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag,
                   precon_thblock, Neuman_itr, independ_nvec, nBlock, *, group=None, boxes=BOXES_THREADS,
                   backend=None):
    """parcel_dcg_ddm's argument list (src/src_DDM/ddm_kernel.f90:2893-2986) on
    torch.distributed; returns (niter, iret).  backend(layout, val, starts, options), when
    given, makes the local operator (parcel_b.dist's spmv / precon interface); the default is
    the GPU library with the process's boxes as its blocks."""
    return _distributed(1, x, b, m, nnd, offset, diaA, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th,
                        ipreflag, itrmax, rtolmax, reshistory, precon_thblock, independ_nvec, group, boxes, backend)


def parcel_dbicgstab_ddm(x, b, m, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim, npe_dim,
                         n_grids, offset_dim, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory,
                         iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, *, group=None,
                         boxes=BOXES_THREADS, backend=None):
    """parcel_dbicgstab_ddm's argument list (ddm_kernel.f90:2988-3080) on torch.distributed."""
    return _distributed(2, x, b, m, nnd, offset, diaA, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th,
                        ipreflag, itrmax, rtolmax, reshistory, precon_thblock, independ_nvec, group, boxes, backend)


def parcel_dgmres_ddm(x, b, m, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim, npe_dim,
                      n_grids, offset_dim, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory,
                      iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, restart, GMRES_GSflag, *,
                      group=None, boxes=BOXES_THREADS, backend=None):
    """parcel_dgmres_ddm's argument list (ddm_kernel.f90:3082-3178) on torch.distributed."""
    return _distributed(3, x, b, m, nnd, offset, diaA, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th,
                        ipreflag, itrmax, rtolmax, reshistory, precon_thblock, independ_nvec, group, boxes, backend,
                        GMRES_m=restart, GMRES_GSflag=GMRES_GSflag)


def parcel_dcagmres_ddm(x, b, m, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim, npe_dim,
                        n_grids, offset_dim, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory,
                        iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep,
                        CAGMRES_basis, CAGMRES_QRflag, *, group=None, boxes=BOXES_THREADS, backend=None):
    """parcel_dcagmres_ddm's argument list (ddm_kernel.f90:3180-3279) on torch.distributed."""
    return _distributed(4, x, b, m, nnd, offset, diaA, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th,
                        ipreflag, itrmax, rtolmax, reshistory, precon_thblock, independ_nvec, group, boxes, backend,
                        CAGMRES_sstep=CAGMRES_sstep, CAGMRES_tstep=CAGMRES_tstep, CAGMRES_basis=CAGMRES_basis,
                        CAGMRES_QRflag=CAGMRES_QRflag)
