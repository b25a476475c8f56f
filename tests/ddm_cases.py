"""General DDM boxes for the tests: any stencil, margin and dimension (the reference's example
only has the 7-point 3D one).  Random nonsymmetric couplings in [-1, 0), zero where the
neighbour leaves the interior (as make_poisson_3D_DDM leaves them at a physical boundary),
a dominant diagonal, b ~ N(0, 1) on the interior.  The dict is oracle/ddm.py's process
description (one process)."""
import itertools

import numpy as np


def star(ndim, reach):
    """Points along the axes up to `reach` cells, plus the centre."""
    pts = [tuple(0 for _ in range(ndim))]
    for d in range(ndim):
        for s in range(1, reach + 1):
            for sg in (-1, 1):
                p = [0] * ndim
                p[d] = sg * s
                pts.append(tuple(p))
    return sorted(pts, key=lambda p: tuple(reversed(p)))


def box(ndim):
    """Every point of the 3^ndim box."""
    return sorted(itertools.product((-1, 0, 1), repeat=ndim), key=lambda p: tuple(reversed(p)))


def stencil_box(n, margin, pts, seed=0):
    ndim = len(n)
    pad = [v + 2 * margin for v in n]
    stride = [1, pad[0], pad[0] * (pad[1] if ndim > 1 else 1)][:ndim]
    m = int(np.prod(pad))
    nnd = len(pts)
    od = np.array(pts, dtype=np.int32)                        # (nnd, ndim)
    offset = (od * np.array(stride)).sum(axis=1).astype(np.int32)
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(v) for v in reversed(n)], indexing="ij")
    coords = [g.ravel() for g in reversed(grids)]             # x fastest
    j = sum((coords[d] + margin) * stride[d] for d in range(ndim))
    val = np.zeros(nnd * m)
    diag = np.zeros(len(j))
    kd = [k for k in range(nnd) if not od[k].any()][0]
    for k in range(nnd):
        if k == kd:
            continue
        inside = np.ones(len(j), bool)
        for d in range(ndim):
            c = coords[d] + od[k, d]
            inside &= (c >= 0) & (c < n[d])
        v = np.where(inside, -rng.uniform(0.1, 1.0, len(j)), 0.0)
        val[k * m + j] = v
        diag += np.abs(v)
    val[kd * m + j] = 1.0 + diag * rng.uniform(1.0, 1.3, len(j))
    b = np.zeros(m)
    b[j] = rng.standard_normal(len(j))
    n3 = list(n) + [1] * (3 - ndim)
    pad3 = pad + [1] * (3 - ndim)
    return dict(val=val, offset=offset, offset_dim=np.asfortranarray(od).ravel(order="F").astype(np.int32),
                b=b, x_exact=np.zeros(m), n=n3, nd=list(n), start=[0, 0, 0], pad=pad3, m=m, margin=margin,
                margins=tuple([margin] * ndim + [0] * (3 - ndim)), rxyz=(0, 0, 0), nnd=nnd)


def split_stencil(gn, npe, rank, margin, pts, seed=0):
    """Process `rank`'s box (set_rank_xyz, set_grids_decompostion) of one global random
    stencil matrix on the grid gn: the same couplings as stencil_box would give the whole grid,
    each process holding its interior rows (couplings into other processes kept, into the
    outside of the grid zero)."""
    import ddm as oddm
    rxyz = oddm.rank_xyz(rank, npe)
    n, start, pad, m = oddm.grids_decomposition(gn, npe, rxyz, margin)
    nnd = len(pts)
    od = np.array(pts, dtype=np.int32)
    stride = [1, pad[0], pad[0] * pad[1]]
    offset = (od * np.array(stride)).sum(axis=1).astype(np.int32)
    rng = np.random.default_rng(seed)
    G = int(np.prod(gn))
    gval = -rng.uniform(0.1, 1.0, (nnd, G))              # coupling of global cell g along point k
    kd = [k for k in range(nnd) if not od[k].any()][0]
    zz, yy, xx = np.meshgrid(*[np.arange(v) for v in reversed(gn)], indexing="ij")
    gx, gy, gz = xx.ravel(), yy.ravel(), zz.ravel()
    inside = np.ones((nnd, G), bool)
    for k in range(nnd):
        for d, c in enumerate((gx, gy, gz)):
            inside[k] &= (c + od[k, d] >= 0) & (c + od[k, d] < gn[d])
    gval = np.where(inside, gval, 0.0)
    gval[kd] = 1.0 + np.abs(np.delete(gval, kd, axis=0)).sum(axis=0) * rng.uniform(1.0, 1.3, G)
    gb = rng.standard_normal(G)
    jz, jy, jx = np.meshgrid(*[np.arange(v) for v in reversed(n)], indexing="ij")
    jx, jy, jz = jx.ravel(), jy.ravel(), jz.ravel()
    g = (jx + start[0]) + gn[0] * ((jy + start[1]) + gn[1] * (jz + start[2]))
    j = (jx + margin) + pad[0] * ((jy + margin) + pad[1] * (jz + margin))
    val = np.zeros(nnd * m)
    for k in range(nnd):
        val[k * m + j] = gval[k, g]
    b = np.zeros(m)
    b[j] = gb[g]
    return dict(val=val, offset=offset, offset_dim=np.asfortranarray(od).ravel(order="F").astype(np.int32),
                b=b, x_exact=np.zeros(m), n=n, start=start, pad=pad, m=m, margin=margin, rxyz=rxyz, nnd=nnd)
