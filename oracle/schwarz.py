"""Additive Schwarz with overlap over processes, restated for the oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the distributed additive
Schwarz preconditioner (parcel_b/schwarz.py), never by the product.

The reference (src/matrix.f90) overlaps every block-Jacobi block of every process:
  * get_AS_region (matrix.f90:3146-3218): block b of a process owns the rows that
    divide_region gives it, and its region reaches addL rows further on both sides (into
    the neighbouring block, or the neighbouring process for the first and last block),
    clipped to row 1 and, past the last row, to the process's own end;
  * check_AS_region (matrix.f90:3220-3287): if some block has fewer than 2 addL rows, the
    whole preconditioner falls back to block Jacobi (addL = 0);
  * get_DILU_DInv_AS_crs (matrix.f90:3809-4375): each region's matrix is the global matrix
    on the region's rows and columns; its D-ILU (ILU_method 1 ILUD or 2 MLUD) is computed on
    it alone;
  * AdditiveSchwarz_crs, AdditiveSchwarz_ILU_crs and AS_Local (matrix.f90:4749-4858,
    5804-6009): the region's right-hand side is r on the whole region (BASIC, RESTRICT; the
    other processes' rows come by set_AS_vec) or r on the block's own rows and zero on the
    rest of the region (INTERPOLATE, NONE); the results are summed over every region that
    covers a row (BASIC, INTERPOLATE; the other processes' shares come by get_AS_vec) or
    taken from the row's own block (RESTRICT, NONE).
On one process the reference runs block Jacobi instead (the CPU side switches the
preconditioner, c_krylov_wrapper.f90:753-756).
"""
from __future__ import annotations

import numpy as np

import oracle

BASIC, RESTRICT, INTERPOLATE, NONE = 1, 2, 3, 4


def divide_region(r, nparts, lo, hi):
    """divide_region (common.f90:125-182): 1-based inclusive part r of [lo, hi]."""
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
    """The process's blocks (0-based global [start, end)) for rows [lo, lo + n)."""
    nb = max(1, min(nb, n))
    out = []
    for b in range(nb):
        a, z = divide_region(b, nb, 1, n)
        out.append((lo + a - 1, lo + z))
    return out


def regions(ranges, nblocks, addL, gn):
    """Every (process, block): (own start, own end, region start, region end), 0-based."""
    out = []
    for (lo, n) in ranges:
        for (olo, ohi) in own_blocks(lo, n, nblocks):
            rlo = max(olo - addL, 0)
            rhi = ohi + addL
            if rhi > gn:
                rhi = lo + n
            out.append((olo, ohi, rlo, rhi))
    return out


def falls_back(ranges, nblocks, addL):
    """check_AS_region: block Jacobi when addL is 0 or some block has fewer than 2 addL rows."""
    if addL <= 0:
        return True
    return any((ohi - olo) // 2 < addL for (lo, n) in ranges for (olo, ohi) in own_blocks(lo, n, nblocks))


def apply(A, ranges, nblocks, addL, iflag, r, ILU_method=1):
    """s = M^-1 r for the global CRS matrix A split into the process row ranges
    [(first row, rows), ...] (0-based, in process order)."""
    import scipy.sparse as sp
    from parcel_b.problems import CRS
    gn = A.n
    S = sp.csr_matrix((A.val, A.col - 1, A.rowptr - 1), shape=(gn, gn))
    r = np.asarray(r, dtype=np.float64)
    if len(ranges) == 1 or falls_back(ranges, nblocks, addL):
        starts = [b[0] for (lo, n) in ranges for b in own_blocks(lo, n, nblocks)] + [gn]
        return oracle.precon_apply(A, r, ipreflag=2, ILU_method=ILU_method, blocks=starts)
    s = np.zeros(gn)
    for (olo, ohi, rlo, rhi) in regions(ranges, nblocks, addL, gn):
        sub = S[rlo:rhi, rlo:rhi].tocsr()
        sub.sort_indices()
        R = CRS(n=rhi - rlo, rowptr=(sub.indptr + 1).astype(np.int32), col=(sub.indices + 1).astype(np.int32),
                val=sub.data.copy())
        rhs = r[rlo:rhi].copy()
        if iflag in (INTERPOLATE, NONE):
            rhs[:olo - rlo] = 0.0
            rhs[ohi - rlo:] = 0.0
        z = oracle.precon_apply(R, rhs, ipreflag=2, ILU_method=ILU_method, blocks=[0, rhi - rlo])
        if iflag in (RESTRICT, NONE):
            s[olo:ohi] = z[olo - rlo:ohi - rlo]
        else:
            s[rlo:rhi] += z
    return s
