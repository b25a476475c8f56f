"""The DDM format split over processes (parcel_b/ddm.py) on CPU processes over gloo.

Four processes (npe = (1, 2, 2) and (2, 2, 1)) each hold their padded box of the example's
DDM Poisson problem (make_poisson_3D_DDM, src/example/ddm_setup.f90:127-345) and call
parcel_dcg_ddm / parcel_dgmres_ddm with a test backend: the product of the process's rows
in numpy and the oracle's D-ILU on its owned boxes.  The decomposition logic is the
product's (global numbering, the margin cells mapped to the neighbours' rows, the halo plan,
the boxes as blocks); the histories must reproduce the oracle's single-process solve of the
same global system (oracle/ddm.py: the rows numbered process by process, box by box) with
the same iteration counts, within 1e-8 relative while the residual is above 1e-8 of its
start (rank-ordered partial sums), and x must land in the interior cells of each box.
Eight processes (npe = (2, 2, 2)) carry a 27-point stencil with random nonsymmetric
couplings cut from one global field, so each process couples to its face, edge and corner
neighbours (all 7 others) through its margin cells.  The library's host-side box numbering
(parcel_b_ddm_order) is checked against the oracle's here too (it needs no GPU)."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GN = (12, 10, 8)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class OracleLocal:
    """Test backend: the process's rows as a scipy matrix over [owned | halo]; the oracle's
    block-Jacobi D-ILU on the owned-owned submatrix with the process's boxes as blocks."""

    def __init__(self, lay, val, starts, options):
        import scipy.sparse as sp
        import torch

        import oracle
        from parcel_b import problems
        rp = lay.rowptr.astype(np.int64) - 1
        ci = lay.local_col.astype(np.int64) - 1
        self.torch = torch
        self.A = sp.csr_matrix((val, ci, rp), shape=(lay.n, lay.n_ext))
        own = self.A[:, :lay.n].tocsr()
        own.sort_indices()
        Aoo = problems.CRS(n=lay.n, rowptr=(own.indptr + 1).astype(np.int32), col=(own.indices + 1).astype(np.int32),
                           val=own.data.astype(np.float64))
        self.M = oracle.Precon(oracle.Matrix(Aoo), ipreflag=options["ipreflag"], ILU_method=1,
                               blocks=np.asarray(starts, np.int64))

    def spmv(self, x_ext, y):
        y.copy_(self.torch.from_numpy(self.A @ x_ext.numpy()))

    def precon(self, r, z):
        z.copy_(self.torch.from_numpy(np.asarray(self.M(r.numpy().copy()), dtype=np.float64)))


def _part(gn, npe, rank, stencil):
    import ddm as oddm
    import ddm_cases
    if stencil == "7":
        return oddm.poisson3d_ddm(gn, npe, rank)
    return ddm_cases.split_stencil(gn, npe, rank, 1, ddm_cases.box(3), seed=5)


def _worker(rank, world, port, npe, solver, boxes, q, gn=GN, stencil="7"):
    try:
        sys.path[:0] = [os.path.join(ROOT, "parcel-legacy_b200"), os.path.join(ROOT, "oracle"), HERE]
        import torch
        import torch.distributed as dist

        from parcel_b import ddm
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        p = _part(gn, npe, rank, stencil)
        x = np.zeros(p["m"])
        hist = np.zeros(500)
        args = (x, p["b"], p["m"], p["nnd"], p["offset"], p["val"], 0, np.zeros(0, np.int32), 1, 3, np.array(npe),
                np.array(p["n"]), p["offset_dim"], 1, 2, 2, 1, 500, 1e-10, hist, 0, 2, 1, -1, 0)
        kw = dict(boxes=boxes, backend=OracleLocal)
        if solver == 1:
            niter, iret = ddm.parcel_dcg_ddm(*args, **kw)
        elif solver == 2:
            niter, iret = ddm.parcel_dbicgstab_ddm(*args, **kw)
        elif solver == 4:
            niter, iret = ddm.parcel_dcagmres_ddm(*args, 4, 3, 1, 5, **kw)   # s, t, Newton, Cholesky QR2
        else:
            niter, iret = ddm.parcel_dgmres_ddm(*args, 10, 1, **kw)
        q.put((rank, niter, iret, hist[:niter].copy(), x))
        dist.destroy_process_group()
    except Exception:
        import traceback
        q.put((rank, "error", traceback.format_exc(), None, None))


@pytest.mark.parametrize("npe,solver,boxes", [((1, 2, 2), 1, 0), ((2, 2, 1), 3, 0), ((1, 2, 2), 1, 1),
                                               ((2, 1, 2), 2, 1), ((2, 2, 1), 4, 1)])
def test_ddm_over_processes_reproduces_the_global_solve(npe, solver, boxes):
    import ddm as oddm
    import oracle
    from parcel_b.problems import CRS
    world = int(np.prod(npe))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, npe, solver, boxes, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
    for o in out:
        assert o[1] != "error", o[2]
    boxes_of = (lambda n: oddm.thread_boxes(n, 1, 2)) if boxes == 0 else oddm.cube_boxes
    parts = [oddm.poisson3d_ddm(GN, npe, r) for r in range(world)]
    G = oddm.global_system(parts, npe, boxes_of)
    A = CRS(n=G["n"], rowptr=G["rowptr"], col=G["col"], val=G["val"])
    if solver == 4:   # CA-GMRES: its own oracle and parity criteria (iterations within 2, 1e-6)
        import cagmres
        xo, ho, no, io = cagmres.pcagmres(A, G["b"], s=4, t=3, basis=1, qrflag=5, itrmax=500, rtolmax=1e-10,
                                          ipreflag=2, ILU_method=1, blocks=G["starts"])
    else:
        kw = dict(solver=solver, ipreflag=2, ILU_method=1, itrmax=500, rtolmax=1e-10, GMRES_m=10, GMRES_GSflag=1)
        xo, ho, no, io = oracle.solve(A, G["b"], blocks=G["starts"], **kw)
    for rank, niter, iret, hist, x in out:
        sel = G["rank"] == rank
        if solver == 4:
            assert iret == io == 0 and abs(niter - no) <= 2, (rank, niter, no)
            k = min(niter, no)
            msk = ho[:k] > 1e-8
            assert np.max(np.abs(hist[:k][msk] - ho[:k][msk]) / ho[:k][msk]) < 1e-6
            assert np.max(np.abs(x[G["padded"][sel]] - xo[sel])) <= 1e-7 * np.max(np.abs(xo))
        else:
            assert (niter, iret) == (no, io), (rank, niter, iret, no, io)
            msk = ho[:niter] > 1e-8 * ho[0]
            assert np.max(np.abs(hist[msk] - ho[:niter][msk]) / ho[:niter][msk]) < 1e-8
            assert np.max(np.abs(x[G["padded"][sel]] - xo[sel])) <= 1e-8 * np.max(np.abs(xo))
        interior = np.zeros(len(x), bool)
        interior[G["padded"][sel]] = True
        assert not x[~interior].any()   # the margin is left as it was


@pytest.mark.parametrize("n,boxes,div,nth", [((9, 8, 7), 0, 1, 4), ((9, 8, 7), 0, 2, 3), ((9, 8, 7), 0, 3, 9),
                                             ((18, 6, 5), 1, 1, -1), ((3, 2, 1), 0, 1, 5)])
def test_library_box_order_is_the_oracle_numbering(n, boxes, div, nth):
    """parcel_b_ddm_order (host-side, no GPU) numbers a box's cells as oracle/ddm.py does."""
    import ddm as oddm
    from parcel_b import ddm
    perm, starts = ddm.order(n, 7, margin=1, div_direc_th=div, boxes=boxes, precon_thblock=nth)
    bx = oddm.thread_boxes(n, div, max(nth, 1)) if boxes == 0 else oddm.cube_boxes(n)
    idx, ost = oddm.box_order(n, bx)
    assert np.array_equal(starts, ost)
    z, y, x = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
    pj = (x + 1) + (n[0] + 2) * ((y + 1) + (n[1] + 2) * (z + 1))
    want = np.empty(int(np.prod(n)), np.int64)
    want[idx.ravel()] = pj.ravel()
    assert np.array_equal(perm, want)


def test_decomposition_rejects_inconsistent_stencils():
    """offset must be offset_dim applied to the padded strides (checked before any exchange)."""
    import ddm as oddm
    p = oddm.poisson3d_ddm((6, 5, 4), (1, 1, 1), 0)
    bad = p["offset"].copy()
    bad[0] += 1
    port = _free_port()
    import torch.distributed as dist

    from parcel_b import ddm
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        with pytest.raises(ValueError):
            ddm.Decomposition(p["val"], bad, p["offset_dim"], p["n"], (1, 1, 1))
        dec = ddm.Decomposition(p["val"], p["offset"], p["offset_dim"], p["n"], (1, 1, 1))
        assert dec.layout.n_ext == dec.n_int == 120 and dec.gn == 120
    finally:
        dist.destroy_process_group()


def test_27_point_stencil_over_eight_processes():
    """A 27-point stencil with random nonsymmetric couplings on a 2 x 2 x 2 process split:
    every process couples to its face, edge and corner neighbours, so the margin cells reach
    all 7 other processes; GMRES against the oracle's global solve."""
    import ddm as oddm
    import oracle
    from parcel_b.problems import CRS
    gn, npe, world = (10, 8, 8), (2, 2, 2), 8
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, npe, 3, 0, q, gn, "27")) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
    for o in out:
        assert o[1] != "error", o[2]
    parts = [_part(gn, npe, r, "27") for r in range(world)]
    G = oddm.global_system(parts, npe, lambda n: oddm.thread_boxes(n, 1, 2))
    xo, ho, no, io = oracle.solve(CRS(n=G["n"], rowptr=G["rowptr"], col=G["col"], val=G["val"]), G["b"],
                                  blocks=G["starts"], solver=3, ipreflag=2, ILU_method=1, itrmax=500,
                                  rtolmax=1e-10, GMRES_m=10, GMRES_GSflag=1)
    for rank, niter, iret, hist, x in out:
        assert (niter, iret) == (no, io), (rank, niter, iret, no, io)
        msk = ho[:niter] > 1e-8 * ho[0]
        assert np.max(np.abs(hist[msk] - ho[:niter][msk]) / ho[:niter][msk]) < 1e-8
        sel = G["rank"] == rank
        assert np.max(np.abs(x[G["padded"][sel]] - xo[sel])) <= 1e-8 * np.max(np.abs(xo))
        interior = np.zeros(len(x), bool)
        interior[G["padded"][sel]] = True
        assert not x[~interior].any()


def test_solve_out_argument_is_checked_before_the_library():
    """out must be float64 with m entries, on the side b is on, and excludes x0."""
    import ddm as oddm
    from parcel_b import ddm
    p = oddm.poisson3d_ddm((6, 5, 4), (1, 1, 1), 0)
    args = (p["val"], p["offset"], p["offset_dim"], p["n"], p["b"])
    with pytest.raises(ValueError):
        ddm.solve(*args, np.zeros(p["m"]), out=np.zeros(p["m"]))
    with pytest.raises((TypeError, ValueError)):
        ddm.solve(*args, out=np.zeros(p["m"], np.float32))
    with pytest.raises((TypeError, ValueError)):
        ddm.solve(*args, out=np.zeros(p["m"] - 1))
