"""Double-double oracle in numpy (TEST INFRASTRUCTURE ONLY).

Restates the reference's dd arithmetic (src/dd_func.f90:5-98: dd_add / dd_sub / dd_mul,
the macro forms in src/ddadd.h and src/ddmul.h) element-wise on float64 arrays.  numpy
evaluates every operation with one IEEE rounding and no contraction, so the order of
operations is the reference's exactly.  residual() follows ddcalc_res_CRS
(src/ddkrylov.f90:1281-1310): r = ddMatVec_crs(A, x) then ddaxpy(1, b, -1, r).
"""
from __future__ import annotations

import numpy as np

SPLIT = 134217729.0


def add(ah, al, bh, bl):
    p1 = ah + bh
    p2 = p1 - ah
    t1l = (ah - (p1 - p2)) + (bh - p2)
    t1h = p1
    t1l = (t1l + al) + bl
    s1 = t1h + t1l
    t1l = t1l - (s1 - t1h)
    return s1, t1l


def mul(ah, al, bh, bl):
    t1h = ah * bh
    u1 = SPLIT * ah
    p1 = u1 - (u1 - ah)
    p2 = ah - p1
    u1 = SPLIT * bh
    r1 = u1 - (u1 - bh)
    r2 = bh - r1
    t1l = (((p1 * r1 - t1h) + p1 * r2) + p2 * r1) + p2 * r2
    t1l = t1l + (ah * bl + al * bh)
    s1 = t1h + t1l
    t1l = t1l - (s1 - t1h)
    return s1, t1l


def residual(A, x_hi, x_lo=None, b_hi=None, b_lo=None):
    """r = b - A x in double-double; A a problems.CRS (1-based), values taken as (a, 0)."""
    n = A.n
    x_lo = np.zeros(n) if x_lo is None else x_lo
    b_lo = np.zeros(n) if b_lo is None else b_lo
    rp = A.rowptr.astype(np.int64) - 1
    lens = np.diff(rp)
    th = np.zeros(n)
    tl = np.zeros(n)
    for k in range(int(lens.max()) if n else 0):
        m = lens > k
        j = rp[:-1][m] + k
        c = A.col[j].astype(np.int64) - 1
        ch, cl = mul(A.val[j], np.zeros(len(j)), x_hi[c], x_lo[c])
        th[m], tl[m] = add(ch, cl, th[m], tl[m])
    bh, bl = mul(np.ones(n), np.zeros(n), b_hi, b_lo)
    ch, cl = mul(-np.ones(n), np.zeros(n), th, tl)
    return add(bh, bl, ch, cl)
