"""The oracle's DIA restatements (crs2dia / dia2crs, src/matrix.f90:7147-7576) on the CPU.

The reference's own DIA solve reproduces its CRS solve on the templates
(template_cpu/STDOUT_run prints identical CRS and DIA histories for CG + D-ILU, 80 blocks,
160^3), so a DIA matrix is pinned by the CRS matrix it stands for: these tests check that
DIA -> CRS gives back exactly the CRS matrix the DIA arrays were made from, whatever the
order of the offsets, and that zeros and out-of-range entries are not part of it.
"""
import numpy as np
import pytest

import oracle
from conftest import poisson_reference
from parcel_b import problems

MATS = {
    "poisson3d_10": lambda: poisson_reference(10)[0],
    "convdiff_9": lambda: problems.convdiff3d_upwind(9),
    "banded_800": lambda: problems.banded_random(800, seed=3),
}


@pytest.mark.parametrize("name", list(MATS))
def test_dia_round_trip_is_exact(name):
    A = MATS[name]()
    dia, off = oracle.crs_to_dia(A)
    assert np.all(np.diff(off) > 0)
    B, _ = oracle.dia_to_crs(dia, off, A.n)
    assert np.array_equal(B.rowptr, A.rowptr) and np.array_equal(B.col, A.col) and np.array_equal(B.val, A.val)
    # the same diagonals in another order describe the same matrix
    p = np.random.default_rng(1).permutation(len(off))
    C, _ = oracle.dia_to_crs(dia.reshape(len(off), A.n)[p].ravel(), off[p], A.n)
    assert np.array_equal(C.col, A.col) and np.array_equal(C.val, A.val)


def test_dia_drops_zeros_and_out_of_range_entries():
    A = problems.convdiff3d_upwind(6)
    dia, off = oracle.crs_to_dia(A)
    d = dia.reshape(len(off), A.n).copy()
    lo = int(np.where(off == -1)[0][0])
    hi = int(np.where(off == off.max())[0][0])
    d[lo, 0] = 7.0            # column 0 - 1: outside the rows
    d[hi, A.n - 1] = -3.0     # column past n
    B, _ = oracle.dia_to_crs(d.ravel(), off, A.n)
    assert np.array_equal(B.col, A.col) and np.array_equal(B.val, A.val)


def test_dia_solve_equals_crs_solve():
    A, b, _ = poisson_reference(12)
    dia, off = oracle.crs_to_dia(A)
    kw = dict(solver=1, ipreflag=2, ILU_method=1, precon_thblock=8, itrmax=500, rtolmax=1e-10)
    x1, h1, n1, i1 = oracle.solve(A, b, **kw)
    x2, h2, n2, i2 = oracle.solve_dia(dia, off, b, **kw)
    assert (n1, i1) == (n2, i2) and np.array_equal(h1, h2) and np.array_equal(x1, x2)


def test_dd_low_parts_follow_their_entries():
    A = problems.convdiff3d_upwind(7)
    alo = A.val * 1e-17
    dia, off = oracle.crs_to_dia(A)
    dlo, _ = oracle.crs_to_dia(A, val=alo)
    B, blo = oracle.dia_to_crs(dia, off, A.n, dia_lo=dlo)
    assert np.array_equal(B.val, A.val) and np.array_equal(blo, alo)
