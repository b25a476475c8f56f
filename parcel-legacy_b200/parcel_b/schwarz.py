"""Additive Schwarz with overlap over processes (ipreflag = 3 in the row-distributed solve).

The reference overlaps every block-Jacobi block of every process by addL rows on both
sides (get_AS_region, src/matrix.f90:3146-3218): the first and last block of a process reach
into the neighbouring processes, the others into the neighbouring blocks.  Each region's
matrix is the global matrix on its rows and columns, with its own D-ILU
(get_DILU_DInv_AS_crs, matrix.f90:3809-4375).  An application (AdditiveSchwarz_crs,
matrix.f90:4749-4858; AdditiveSchwarz_ILU_crs and AS_Local, 5804-6009) solves every region
from r on the region (BASIC, RESTRICT: the neighbours' boundary rows of r arrive first) or r
on the block's own rows and zero elsewhere (INTERPOLATE, NONE), then either sums the regions'
results over every row they cover (BASIC, INTERPOLATE: the neighbours' shares of this
process's rows arrive last) or keeps each block's own rows (RESTRICT, NONE).  If some block
has fewer than 2 addL rows the reference falls back to block Jacobi (check_AS_region,
matrix.f90:3220-3287), and so does this; on one process it runs block Jacobi.

Here the regions of a process are laid out one after another as the blocks of one expanded
matrix (overlapping rows appear in each region that covers them), so one block-Jacobi D-ILU
application of the library (parcel_b_local_create_blocks, the regions as explicit blocks)
solves all of them; a gather builds the expanded right-hand side and a scatter (or a
scatter-add: a row is covered by at most two regions, so the sum does not depend on the
order) brings the result back.  The boundary rows of the matrix come from the neighbours
once, at set-up; each application exchanges addL values with each neighbour before (BASIC,
RESTRICT) and after (BASIC, INTERPOLATE) the local solve.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

BASIC, RESTRICT, INTERPOLATE, NONE = 1, 2, 3, 4


def divide_region(r, nparts, lo, hi):
    """divide_region (src/common.f90:125-182): 1-based inclusive part r of [lo, hi]."""
    if hi == lo:
        return lo, hi
    region = hi - lo + 1
    blk, over = region // nparts, region % nparts
    if r < over:
        a = lo + blk * r + r
        return a, a + blk
    a = lo + blk * r + over
    return a, a + blk - 1


def own_blocks(lo, n, nb):
    """The blocks of the rows [lo, lo + n) (0-based global [start, end))."""
    nb = max(1, min(nb, n))
    return [(lo + a - 1, lo + z) for a, z in (divide_region(b, nb, 1, n) for b in range(nb))]


class _Rows:
    """Rows as (rowptr from 0, global columns 0-based, values)."""

    def __init__(self, rp, col, val):
        self.rp, self.col, self.val = np.asarray(rp, np.int64), np.asarray(col, np.int64), np.asarray(val, np.float64)

    def take(self, a, b):
        k0, k1 = self.rp[a], self.rp[b]
        return _Rows(self.rp[a:b + 1] - k0, self.col[k0:k1], self.val[k0:k1])


class Schwarz:
    """The overlapped additive Schwarz preconditioner of this process.

    layout: the process's dist.Layout; rowptr (1-based), col (global, 1-based), val: its rows;
    nblocks, addL, iflagAS, ILU_method: the options; make_precon(n, rowptr, col, val, starts,
    options) builds the local block-Jacobi operator of the expanded matrix (rowptr and col
    1-based, local), returning an object with precon(r, z)."""

    def __init__(self, layout, rowptr, col, val, nblocks, addL, iflagAS, ILU_method, make_precon, options):
        self.lay = layout
        self.group = layout.group
        self.iflag = int(iflagAS) if int(iflagAS) in (BASIC, RESTRICT, INTERPOLATE, NONE) else BASIC
        if int(ILU_method) not in (1, 2):
            raise ValueError("the overlapped additive Schwarz solves its regions with D-ILU (ILU_method 1 or 2)")
        rank, world = layout.rank, layout.world
        gn = layout.gn
        lo, n = layout.istart - 1, layout.n
        blocks = own_blocks(lo, n, nblocks)
        short = 1 if any((b - a) // 2 < addL for a, b in blocks) or addL <= 0 else 0
        flags = [None] * world
        dist.all_gather_object(flags, short, group=self.group)
        self.bj = world == 1 or any(flags)           # check_AS_region: block Jacobi for everyone
        rows = _Rows(np.asarray(rowptr, np.int64) - 1, np.asarray(col, np.int64) - 1, val)
        opts = dict(options, ipreflag=2, ILU_method=int(ILU_method))
        if self.bj:
            self.addL = 0
            starts = [a - lo for a, _ in blocks] + [n]
            self.M = make_precon(n, *self._local(rows, lo, n, lo, lo + n), starts, opts)
            return
        self.addL = addL
        # the neighbours' boundary rows (addL each), with global columns
        mine = (rows.take(0, addL), rows.take(n - addL, n))
        edges = [None] * world
        dist.all_gather_object(edges, mine, group=self.group)
        self.prev = rank - 1 if rank > 0 else None
        self.next = rank + 1 if rank < world - 1 else None
        elo = lo - addL if self.prev is not None else lo
        ehi = lo + n + addL if self.next is not None else lo + n
        parts = ([edges[self.prev][1]] if self.prev is not None else []) + [rows] + \
                ([edges[self.next][0]] if self.next is not None else [])
        rp, cl, vl, off = [0], [], [], 0
        for p in parts:
            rp.extend((p.rp[1:] + off).tolist())
            off += len(p.col)
            cl.append(p.col)
            vl.append(p.val)
        ext = _Rows(rp, np.concatenate(cl), np.concatenate(vl))
        self.elo, self.ehi, self.lo = elo, ehi, lo
        # regions (get_AS_region) in the extended numbering, laid out one after another
        gmap, own_src, own_dst, mask, starts = [], [], [], [], [0]
        erp, ecol, eval_ = [0], [], []
        for (olo, ohi) in blocks:
            rlo = max(olo - addL, 0)
            rhi = ohi + addL
            if rhi > gn:
                rhi = lo + n
            base = starts[-1]
            for g in range(rlo, rhi):
                k0, k1 = ext.rp[g - elo], ext.rp[g - elo + 1]
                c = ext.col[k0:k1]
                keep = (c >= rlo) & (c < rhi)
                ecol.append(c[keep] - rlo + base)
                eval_.append(ext.val[k0:k1][keep])
                erp.append(erp[-1] + int(keep.sum()))
            gmap.extend(range(rlo - elo, rhi - elo))
            m = np.zeros(rhi - rlo, bool)
            m[olo - rlo:ohi - rlo] = True
            mask.append(m)
            own_src.extend(range(base + olo - rlo, base + ohi - rlo))
            own_dst.extend(range(olo - lo, ohi - lo))
            starts.append(base + rhi - rlo)
        nexp = starts[-1]
        ecol = np.concatenate(ecol)
        self.M = make_precon(nexp, np.asarray(erp, np.int32) + 1, ecol.astype(np.int32) + 1, np.concatenate(eval_),
                             starts, opts)
        self.gmap_np = np.asarray(gmap, np.int64)
        self.own_src_np = np.asarray(own_src, np.int64)
        self.own_dst_np = np.asarray(own_dst, np.int64)
        self.mask_np = np.concatenate(mask)
        self.nexp = nexp
        self._dev = None

    @staticmethod
    def _local(rows, lo, n, a, b):
        """Rows [a, b) with columns restricted to [a, b), renumbered from 1."""
        r = rows.take(a - lo, b - lo)
        keep = (r.col >= a) & (r.col < b)
        rp = np.concatenate([[0], np.cumsum([int(keep[r.rp[i]:r.rp[i + 1]].sum()) for i in range(b - a)])])
        return (rp + 1).astype(np.int32), (r.col[keep] - a + 1).astype(np.int32), r.val[keep]

    def _on(self, dev):
        if self._dev != dev:
            t = lambda a: torch.from_numpy(a).to(dev)
            self.gmap, self.own_src, self.own_dst = t(self.gmap_np), t(self.own_src_np), t(self.own_dst_np)
            self.mask = t(self.mask_np)
            self.rexp = torch.zeros(self.nexp, dtype=torch.float64, device=dev)
            self.zexp = torch.zeros(self.nexp, dtype=torch.float64, device=dev)
            self.vext = torch.zeros(self.ehi - self.elo, dtype=torch.float64, device=dev)
            self._dev = dev

    def _swap(self, send_prev, send_next, recv_prev, recv_next):
        """addL values each way with the neighbouring processes (one batched exchange)."""
        ops = []
        if self.prev is not None:
            ops.append(dist.P2POp(dist.isend, send_prev.contiguous(), self.prev, group=self.group))
            ops.append(dist.P2POp(dist.irecv, recv_prev, self.prev, group=self.group))
        if self.next is not None:
            ops.append(dist.P2POp(dist.isend, send_next.contiguous(), self.next, group=self.group))
            ops.append(dist.P2POp(dist.irecv, recv_next, self.next, group=self.group))
        if ops:
            for q in dist.batch_isend_irecv(ops):
                q.wait()

    def precon(self, r, z):
        if self.bj:
            self.M.precon(r, z)
            return
        self._on(r.device)
        L, n = self.addL, self.lay.n
        a = self.lo - self.elo                        # rows of the previous process in the extension
        v = self.vext
        v.zero_()
        v[a:a + n] = r
        if self.iflag in (BASIC, RESTRICT):           # set_AS_vec: the neighbours' boundary rows of r
            self._swap(r[:L], r[n - L:], v[:a], v[a + n:])
        torch.index_select(v, 0, self.gmap, out=self.rexp)
        if self.iflag in (INTERPOLATE, NONE):
            self.rexp.mul_(self.mask)
        self.M.precon(self.rexp, self.zexp)
        if self.iflag in (RESTRICT, NONE):
            z.index_copy_(0, self.own_dst, self.zexp.index_select(0, self.own_src))
            return
        v.zero_()
        v.index_add_(0, self.gmap, self.zexp)        # AS_Local: the regions' shares, summed
        z.copy_(v[a:a + n])
        if self.prev is not None or self.next is not None:   # get_AS_vec: the neighbours' shares
            from_prev = torch.zeros(L, dtype=torch.float64, device=r.device)
            from_next = torch.zeros(L, dtype=torch.float64, device=r.device)
            self._swap(v[:a], v[a + n:], from_prev, from_next)
            if self.prev is not None:
                z[:L] += from_prev
            if self.next is not None:
                z[n - L:] += from_next
