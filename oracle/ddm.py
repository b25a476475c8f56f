"""DDM stencil format, restated for the oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ (never by the product) as the checker of the
DDM entry points.

A DDM matrix is one process's box of a structured grid padded by `margin` cells per side,
x fastest, with nnd stencil points: diaA[k m + j] couples cell j with cell j + offset[k]
(src/example/ddm_setup.f90).  Restated here:
  * rank_xyz / grids_decomposition: set_rank_xyz and set_grids_decompostion
    (ddm_setup.f90:52-125), every process's interior box;
  * poisson3d_ddm: make_poisson_3D_DDM (ddm_setup.f90:127-345), the example's 7-point
    problem on one process's padded box;
  * thread_boxes: set_region_for_threads (src/common.f90:266-303), the CPU build's slabs;
    cube_boxes: init_DILU_DDM with n/4 divisions per axis (src/src_DDM/precon_ddm_GPU.f90:
    2923-3097, called at ddm_kernel.f90:1009-1017), the CUDA build's boxes;
  * dilu_apply: the D-ILU diagonal of as_ddm_init (src/src_DDM/init_ddm_mod.f90:370-642)
    and the sweeps of ilu_ddm_case_{x,y,z}div without ILUindepend
    (src/src_DDM/aslu_ddm.f90:323-1558), cell by cell on the padded box (small boxes);
  * global_system: the whole grid's matrix with the rows numbered process by process, box
    by box, lexicographically inside a box, and the boxes' row starts, for the CRS oracle
    (oracle.solve(blocks=...)), which reproduces the reference's stored DDM outputs.
"""
from __future__ import annotations

import numpy as np

# make_poisson_3D_DDM's stencil: (x, y, z) offsets in the order of diaA
STENCIL7 = [(0, 0, -1), (0, -1, 0), (-1, 0, 0), (0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]


def rank_xyz(rank, npe):
    """set_rank_xyz: rank = npe_x npe_y rz + npe_x ry + rx."""
    px, py, _ = npe
    return (rank % (px * py)) % px, (rank % (px * py)) // px, rank // (px * py)


def grids_decomposition(gn, npe, rxyz, margin=1):
    """set_grids_decompostion: interior cells per axis (the last process of an axis takes the
    remainder), 0-based first global cell per axis, padded sizes and m."""
    n, start, pad = [], [], []
    for d in range(3):
        n1 = gn[d] // npe[d]
        n2 = gn[d] - n1 * npe[d]
        n.append(n1 + (n2 if rxyz[d] == npe[d] - 1 else 0))
        start.append(n1 * rxyz[d])
        pad.append(n[-1] + 2 * margin)
    return n, start, pad, int(np.prod(pad))


def poisson3d_ddm(gn, npe, rank, margin=1):
    """make_poisson_3D_DDM for process `rank`: diaA (7 m), offset (7), offset_dim (7 x 3,
    column-major as offset_dim(nnd, ndim)), b and the exact solution (m, margin zero)."""
    rx, ry, rz = rxyz = rank_xyz(rank, npe)
    n, start, pad, m = grids_decomposition(gn, npe, rxyz, margin)
    nx, ny, nz = n
    mx, my, _ = pad
    jz, jy, jx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    jx, jy, jz = jx.ravel(), jy.ravel(), jz.ravel()
    j = (jx + margin) + mx * (jy + margin) + mx * my * (jz + margin)
    px, py, pz = npe
    conds = [(rz > 0) | (jz > 0), (ry > 0) | (jy > 0), (rx > 0) | (jx > 0), np.ones(j.shape, bool),
             (rx < px - 1) | (jx < nx - 1), (ry < py - 1) | (jy < ny - 1), (rz < pz - 1) | (jz < nz - 1)]
    val = np.zeros(7 * m)
    for k, c in enumerate(conds):
        val[k * m + j] = np.where(c, -6.0 if k == 3 else 1.0, 0.0)
    od = np.array(STENCIL7, dtype=np.int32)                      # (7, 3)
    offset = (mx * my * od[:, 2] + mx * od[:, 1] + od[:, 0]).astype(np.int32)
    hx, hy, hz = (1.0 / (g + 1) for g in gn)
    ix, iy, iz = jx + start[0], jy + start[1], jz + start[2]
    X, Y, Z = (ix + 1.0) ** 2, (iy + 1.0) ** 2, (iz + 1.0) ** 2
    b = np.zeros(m)
    b[j] = 2.0 * hx ** 2 * hy ** 2 * hz ** 2 * (X * Y + Y * Z + Z * X)
    if rx == px - 1:
        s = jx == nx - 1
        b[j[s]] -= (hy * (iy[s] + 1)) ** 2 * (hz * (iz[s] + 1)) ** 2
    if ry == py - 1:
        s = jy == ny - 1
        b[j[s]] -= (hx * (ix[s] + 1)) ** 2 * (hz * (iz[s] + 1)) ** 2
    if rz == pz - 1:
        s = jz == nz - 1
        b[j[s]] -= (hx * (ix[s] + 1)) ** 2 * (hy * (iy[s] + 1)) ** 2
    xe = np.zeros(m)
    xe[j] = hx ** 2 * hy ** 2 * hz ** 2 * X * Y * Z
    return dict(val=val, offset=offset, offset_dim=np.asfortranarray(od).ravel(order="F").astype(np.int32),
                b=b, x_exact=xe, n=n, start=start, pad=pad, m=m, margin=margin, rxyz=rxyz, nnd=7)


def thread_boxes(n, div_dir, nthreads):
    """set_region_for_threads along axis div_dir (1 x, 2 y, 3 z): thread t gets
    [n1 t, n1 t + n1), n1 = n_d // nthreads, the last thread the rest; empty slabs dropped.
    Boxes as ((x0, x1), (y0, y1), (z0, z1))."""
    d = div_dir - 1
    n1 = n[d] // nthreads
    out = []
    for t in range(nthreads):
        lo = n1 * t
        hi = n[d] if t == nthreads - 1 else lo + n1
        if hi > lo:
            box = [(0, n[0]), (0, n[1]), (0, n[2])]
            box[d] = (lo, hi)
            out.append(tuple(box))
    return out


def cube_boxes(n):
    """init_DILU_DDM with max(n_d // 4, 1) divisions per axis, ceil(n_d / div) cells each
    (the last shorter), boxes ordered z, y, x."""
    div = [max(v // 4, 1) for v in n]
    ln = [n[d] // div[d] + (1 if n[d] % div[d] else 0) for d in range(3)]
    rng = [[(ln[d] * i, min(n[d], ln[d] * (i + 1))) for i in range(div[d])] for d in range(3)]
    return [(bx, by, bz) for bz in rng[2] for by in rng[1] for bx in rng[0]
            if bx[1] > bx[0] and by[1] > by[0] and bz[1] > bz[0]]


def box_order(n, boxes):
    """Local row numbering: idx[z, y, x] = row of interior cell (x, y, z), rows numbered box by
    box, lexicographically (x fastest) inside a box; and the boxes' first rows + total."""
    idx = np.full((n[2], n[1], n[0]), -1, dtype=np.int64)
    starts, r = [], 0
    for (x0, x1), (y0, y1), (z0, z1) in boxes:
        starts.append(r)
        cnt = (x1 - x0) * (y1 - y0) * (z1 - z0)
        idx[z0:z1, y0:y1, x0:x1] = (r + np.arange(cnt)).reshape(z1 - z0, y1 - y0, x1 - x0)
        r += cnt
    starts.append(r)
    assert (idx >= 0).all()
    return idx, np.array(starts, dtype=np.int64)


def dilu_apply(dd, boxes, r, split_axis=None):
    """The DDM block-Jacobi D-ILU applied to r (padded, m entries), on the padded box.

    Diagonal (as_ddm_init): Dinv(j) = a_jj; walking each box lexicographically,
    Dinv(j) <- 1 / Dinv(j), then every upper neighbour k = j + offset(ip) inside the box gets
    Dinv(k) -= a(j, k) a(k, j) Dinv(j).  Sweeps (ilu_ddm_case_*div): forward
    vec2(j) = Dinv(j) (r(j) - sum_lower a vec2), backward vec2(j) -= Dinv(j) sum_upper a vec2,
    vec2 zero on the margin.  split_axis (0, 1, 2) restates the CPU build's slab sweeps, which
    test only that axis against the slab bounds (other axes reach the margin, where vec2 is
    zero); None drops every coupling that leaves the box (the CUDA build's boxes, and the
    block-Jacobi form the product follows).  The two agree for stencils along the
    axes; with diagonal points the split-axis test lets a lower coupling reach into the next
    slab, a cell that another OpenMP thread of the reference is writing at the same time (a
    race there), so the box-restricted form is the one the product follows."""
    val, off, m = dd["val"], dd["offset"], dd["m"]
    nnd = len(off)
    od = np.asarray(dd["offset_dim"]).reshape(3, nnd).T
    mg = dd["margin"]
    mx, my, _ = dd["pad"]
    idiag = int(np.nonzero(off == 0)[0][0])
    lower = [k for k in range(nnd) if off[k] < 0]
    upper = [k for k in range(nnd) if off[k] > 0]

    def pidx(x, y, z):
        return (x + mg) + mx * ((y + mg) + my * (z + mg))

    Dinv = np.ones(m)
    z_ = np.zeros(m)
    for box in boxes:
        (x0, x1), (y0, y1), (z0, z1) = box
        lo, hi = (x0, y0, z0), (x1, y1, z1)
        cells = [(x, y, z) for z in range(z0, z1) for y in range(y0, y1) for x in range(x0, x1)]
        for (x, y, z) in cells:
            Dinv[pidx(x, y, z)] = val[idiag * m + pidx(x, y, z)]
        for (x, y, z) in cells:
            j = pidx(x, y, z)
            Dinv[j] = 1.0 / Dinv[j]
            for ip in upper:
                c = (x + od[ip, 0], y + od[ip, 1], z + od[ip, 2])
                if any(c[d] < lo[d] or c[d] > hi[d] - 1 for d in range(3)):
                    continue
                k = j + off[ip]
                ipp = int(np.nonzero(off == -off[ip])[0][0])
                Dinv[k] = Dinv[k] - val[ip * m + j] * val[ipp * m + k] * Dinv[j]

        def outside(c, d_lo_hi):
            if split_axis is None:   # the box: both bounds on every axis
                return any(c[d] < lo[d] or c[d] > hi[d] - 1 for d in range(3))
            return d_lo_hi(c, split_axis)

        for (x, y, z) in cells:
            j = pidx(x, y, z)
            s = 0.0
            for ip in lower:
                c = (x + od[ip, 0], y + od[ip, 1], z + od[ip, 2])
                if outside(c, lambda c, d: c[d] < lo[d]):
                    continue
                s = s + val[ip * m + j] * z_[j + off[ip]]
            z_[j] = Dinv[j] * (r[j] - s)
        for (x, y, z) in reversed(cells):
            j = pidx(x, y, z)
            s = 0.0
            for ip in upper:
                c = (x + od[ip, 0], y + od[ip, 1], z + od[ip, 2])
                if outside(c, lambda c, d: c[d] > hi[d] - 1):
                    continue
                s = s + val[ip * m + j] * z_[j + off[ip]]
            z_[j] = z_[j] - Dinv[j] * s
    return z_


def global_system(parts, npe, boxes_of):
    """The global matrix of a DDM decomposition, numbered process by process (rank order), box
    by box, lexicographically inside a box.  parts[rank]: the process's DDM dict (as
    poisson3d_ddm returns, with 'n', 'start', 'pad', 'margin', 'val', 'offset_dim'; optional
    'margins' per axis, 0 past ndim, with offset_dim then holding ndim columns);
    boxes_of(n) -> that process's boxes.  Couplings to cells outside the global grid and
    zero values are left out.  Returns (rowptr, col (1-based, sorted), val, b, x_exact,
    starts of every box, the padded index of each row, the rank of each row)."""
    import scipy.sparse as sp
    world = len(parts)
    idx, starts, base = [], [], [0]
    for p in parts:
        i, s = box_order(p["n"], boxes_of(p["n"]))
        idx.append(i)
        starts.append(s[:-1] + base[-1])
        base.append(base[-1] + int(s[-1]))
    N = base[-1]
    gn = [0, 0, 0]
    for d in range(3):
        gn[d] = max(p["start"][d] + p["n"][d] for p in parts)
    owner = np.empty((gn[2], gn[1], gn[0]), dtype=np.int64)
    gidx = np.empty((gn[2], gn[1], gn[0]), dtype=np.int64)
    for r, p in enumerate(parts):
        (sx, sy, sz), (nx, ny, nz) = p["start"], p["n"]
        owner[sz:sz + nz, sy:sy + ny, sx:sx + nx] = r
        gidx[sz:sz + nz, sy:sy + ny, sx:sx + nx] = base[r] + idx[r]
    rows, cols, vals = [], [], []
    b = np.zeros(N)
    xe = np.zeros(N)
    pj = np.zeros(N, dtype=np.int64)
    prank = np.zeros(N, dtype=np.int64)
    for r, p in enumerate(parts):
        (sx, sy, sz), (nx, ny, nz) = p["start"], p["n"]
        (mx, my, _), m = p["pad"], p["m"]
        mgx, mgy, mgz = p.get("margins", (p["margin"],) * 3)   # per axis (0 past ndim)
        nnd = len(p["offset"])
        od = np.asarray(p["offset_dim"]).reshape(-1, nnd).T
        od = np.concatenate([od, np.zeros((nnd, 3 - od.shape[1]), od.dtype)], axis=1)
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        row = base[r] + idx[r]
        j = (xx + mgx) + mx * ((yy + mgy) + my * (zz + mgz))
        b[row.ravel()] = p["b"][j.ravel()]
        xe[row.ravel()] = p["x_exact"][j.ravel()]
        pj[row.ravel()] = j.ravel()
        prank[row.ravel()] = r
        for k in range(nnd):
            gx, gy, gz = xx + sx + od[k, 0], yy + sy + od[k, 1], zz + sz + od[k, 2]
            v = p["val"][k * m + j]
            ok = (gx >= 0) & (gx < gn[0]) & (gy >= 0) & (gy < gn[1]) & (gz >= 0) & (gz < gn[2]) & (v != 0.0)
            rows.append(row[ok])
            cols.append(gidx[gz[ok], gy[ok], gx[ok]])
            vals.append(v[ok])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    A.sort_indices()
    return dict(rowptr=(A.indptr + 1).astype(np.int32), col=(A.indices + 1).astype(np.int32),
                val=A.data.astype(np.float64), n=N, b=b, x_exact=xe,
                starts=np.concatenate(starts + [np.array([N])]).astype(np.int64), padded=pj, rank=prank)
