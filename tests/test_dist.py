"""The row-distributed solve (parcel_b/dist.py) on CPU processes over gloo: CG, BiCGStab
and GMRES.

Two (and three) processes split the rows of a matrix contiguously at block-Jacobi block
boundaries; each runs the distributed recurrences with a test backend: its local product
in numpy and its block-Jacobi ILU(0) from the oracle on its owned-owned submatrix.  The
histories must reproduce the single-process oracle solve with the same blocks (the inner
products sum the per-process partials in rank order, so they differ from one process's
order by round-off only, which grows as the residual falls: 1e-8 relative while the
residual is above 1e-8 of its start, against the 1e-6 of the solver parity tests),
with the same iteration counts and return codes.  This covers the host logic of the
decomposition (layout, halo plan, exchange, reductions, recurrences); the GPU backend runs
in tests/test_gpu_dist.py."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class NumpyLocal:
    """Test backend: the process's rows as a scipy matrix over [owned | halo] and the
    oracle's block-Jacobi ILU on the owned-owned submatrix."""

    def __init__(self, lay, val, nblocks, ipreflag):
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
        self.M = oracle.Precon(oracle.Matrix(Aoo), ipreflag=ipreflag, ILU_method=0, precon_thblock=nblocks)

    def spmv(self, x_ext, y):
        y.copy_(self.torch.from_numpy(self.A @ x_ext.numpy()))

    def precon(self, r, z):
        z.copy_(self.torch.from_numpy(np.asarray(self.M(r.numpy().copy()), dtype=np.float64)))


def _problem(kind):
    from parcel_b import problems
    if kind == "cg":
        A, b, _ = problems.poisson3d_reference(12, 12, 12)
        return A, b, dict(solver=1, itrmax=500, rtolmax=1e-9)
    A = problems.convdiff3d_upwind(12)
    b = problems.rhs_normal(A.n, 3)
    if kind == "bicgstab":
        return A, b, dict(solver=2, itrmax=500, rtolmax=1e-10)
    if kind == "gmres-cgs":
        return A, b, dict(solver=3, itrmax=500, rtolmax=1e-10, GMRES_m=10, GMRES_GSflag=2)
    if kind == "gmres-pj":   # point Jacobi
        return A, b, dict(solver=3, itrmax=800, rtolmax=1e-10, GMRES_m=10, GMRES_GSflag=1)
    if kind.startswith("cagmres"):   # cagmres-s-t-basis-qr
        _, sst, tst, bas, qr = kind.split("-")
        return A, b, dict(solver=4, itrmax=500, rtolmax=1e-10, CAGMRES_sstep=int(sst), CAGMRES_tstep=int(tst),
                          CAGMRES_basis=int(bas), CAGMRES_QRflag=int(qr))
    return A, b, dict(solver=3, itrmax=500, rtolmax=1e-10, GMRES_m=10, GMRES_GSflag=1)


def _worker(rank, world, port, kind, nblocks, q):
    try:
        sys.path[:0] = [os.path.join(ROOT, "parcel-legacy_b200"), os.path.join(ROOT, "oracle")]
        import torch
        import torch.distributed as dist

        from parcel_b import dist as pdist
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        A, b, kw = _problem(kind)
        per = A.n // world                         # block boundaries: n and nblocks divide evenly
        lo, hi = rank * per, (rank + 1) * per
        rp = A.rowptr[lo:hi + 1] - A.rowptr[lo] + 1
        k0, k1 = A.rowptr[lo] - 1, A.rowptr[hi] - 1
        lay = pdist.Layout(hi - lo, A.n, lo + 1, rp, A.col[k0:k1])
        be = NumpyLocal(lay, A.val[k0:k1], nblocks // world, 1 if kind == "gmres-pj" else 2)
        x = torch.zeros(hi - lo, dtype=torch.float64)
        niter, iret, hist = pdist.solve(lay, A.val[k0:k1], torch.from_numpy(b[lo:hi].copy()), x, backend=be, **kw)
        q.put((rank, niter, iret, hist, x.numpy(), lay.n_ext - lay.n))
        dist.destroy_process_group()
    except Exception as e:  # pragma: no cover - reported to the parent
        import traceback
        q.put((rank, "error", traceback.format_exc(), None, None, None))


def _run(kind, world, nblocks):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, nblocks, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    for o in out:
        assert o[1] != "error", o[2]
    return sorted(out, key=lambda o: o[0])


@pytest.mark.parametrize("kind,world", [("cg", 2), ("bicgstab", 2), ("bicgstab", 3), ("gmres", 2), ("gmres", 3),
                                        ("gmres-cgs", 2), ("gmres-pj", 3)])
def test_distributed_solve_reproduces_single_process_history(kind, world):
    import oracle
    nblocks = 2 * world
    A, b, kw = _problem(kind)
    if A.n % world or (A.n // world) % (nblocks // world):
        pytest.skip("rows do not split evenly")
    pre = dict(ipreflag=1) if kind == "gmres-pj" else dict(ipreflag=2, ILU_method=0, precon_thblock=nblocks)
    xo, ho, no, io = oracle.solve(A, b, **pre, **kw)
    out = _run(kind, world, nblocks)
    for rank, niter, iret, hist, x, nhalo in out:
        assert (niter, iret) == (no, io), (rank, niter, iret, no, io)
        m = ho[:niter] > 1e-8 * ho[0]
        assert np.max(np.abs(hist[m] - ho[:niter][m]) / ho[:niter][m]) < 1e-8
        assert nhalo > 0
    x = np.concatenate([o[4] for o in out])
    assert np.max(np.abs(x - xo)) <= 1e-8 * np.max(np.abs(xo))


@pytest.mark.parametrize("kind,world", [("cagmres-4-1-0-4", 2), ("cagmres-4-2-0-5", 3), ("cagmres-2-4-0-3", 2),
                                        ("cagmres-4-3-1-5", 2), ("cagmres-8-2-1-3", 3)])
def test_distributed_cagmres_reproduces_the_oracle(kind, world):
    """CA-GMRES(s, t) over processes (monomial and Newton bases; Cholesky QR, Cholesky QR2 and
    TSQR) against the oracle's CA-GMRES on one process, at its parity criteria: iterations
    within 2, histories within 1e-6 above 1e-8, and the final true residual."""
    import cagmres
    import oracle
    nblocks = 2 * world
    A, b, kw = _problem(kind)
    if A.n % world or (A.n // world) % (nblocks // world):
        pytest.skip("rows do not split evenly")
    xo, ho, no, io = cagmres.pcagmres(A, b, s=kw["CAGMRES_sstep"], t=kw["CAGMRES_tstep"], basis=kw["CAGMRES_basis"],
                                      qrflag=kw["CAGMRES_QRflag"], itrmax=kw["itrmax"], rtolmax=kw["rtolmax"],
                                      ipreflag=2, ILU_method=0, precon_thblock=nblocks)
    out = _run(kind, world, nblocks)
    x = np.concatenate([o[4] for o in out])
    for rank, niter, iret, hist, _, nhalo in out:
        assert iret == io == 0 and abs(niter - no) <= 2, (rank, niter, no)
        k = min(len(ho), len(hist))
        m = ho[:k] > 1e-8
        assert np.max(np.abs(hist[:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6
        assert nhalo > 0
    assert oracle.true_relres(A, b, x) < 1e-9


def test_cagmres_dense_steps_match_the_oracle():
    """The distributed CA-GMRES's host steps (Leja ordering of Ritz values with complex pairs,
    Newton change-of-basis matrix, Hessenberg block update) against the oracle's on random
    inputs."""
    import cagmres

    from parcel_b import dist as pdist
    rng = np.random.default_rng(11)
    for trial in range(20):
        s = int(rng.integers(2, 9))
        H = rng.standard_normal((s, s))
        ev = np.linalg.eigvals(H)
        a = pdist._leja(ev.real, ev.imag)
        b = cagmres.leja(ev.real, ev.imag)
        assert np.allclose(a[0], b[0], rtol=1e-13, atol=0) and np.allclose(a[1], b[1], rtol=1e-13, atol=0), trial
        B1a, B1b = np.zeros((s + 1, s)), np.zeros((s + 1, s))
        for i in range(s):
            B1a[i + 1, i] = B1b[i + 1, i] = 1.0
        pdist._newton_basis(s, B1a, a[0], a[1])
        cagmres.newton_basis(s, B1b, b[0], b[1])
        assert np.array_equal(B1a, B1b)
        # Hessenberg blocks k = 1 and k = 2 from random triangular factors
        t = 2
        R1 = np.triu(rng.standard_normal((s + 1, s + 1))) + 3 * np.eye(s + 1)
        Rk = np.triu(rng.standard_normal((s, s))) + 3 * np.eye(s)
        BRup = rng.standard_normal((s + 1, s + 1))
        Ha, Hb = np.zeros((s * t + 1, s * t)), np.zeros((s * t + 1, s * t))
        ha = pdist._hessenberg_update(s, 1, B1a, Ha, R1, None, None, 0.0)
        hb = cagmres.hessenberg_update(s, t, 1, B1b, Hb, R1, None, None, 0.0)
        ha = pdist._hessenberg_update(s, 2, B1a, Ha, R1, Rk, BRup, ha)
        hb = cagmres.hessenberg_update(s, t, 2, B1b, Hb, R1, Rk, BRup, hb)
        assert np.allclose(Ha, Hb, rtol=1e-12, atol=1e-12 * np.abs(Hb).max()) and np.isclose(ha, hb, rtol=1e-13)


def _dia_worker(rank, world, port, kind, nblocks, q):
    try:
        sys.path[:0] = [os.path.join(ROOT, "parcel-legacy_b200"), os.path.join(ROOT, "oracle")]
        import torch
        import torch.distributed as dist

        import oracle
        from parcel_b import dist as pdist
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        A, b, kw = _problem(kind[4:])
        dia, off = oracle.crs_to_dia(A)
        off = off[::-1].copy()                     # any offset order
        dia = dia.reshape(len(off), A.n)[::-1]
        per = A.n // world
        lo, hi = rank * per, (rank + 1) * per
        mine = np.ascontiguousarray(dia[:, lo:hi]).ravel()
        x = torch.zeros(hi - lo, dtype=torch.float64)
        hist = np.zeros(kw["itrmax"] + 2)
        be = lambda lay, val, opts: NumpyLocal(lay, val, nblocks // world, 2)
        common = dict(ipreflag=2, ILU_method=0, addL=0, iflagAS=1, itrmax=kw["itrmax"], rtolmax=kw["rtolmax"],
                      reshistory=hist, backend=be)
        args = (x, torch.from_numpy(b[lo:hi].copy()), hi - lo, A.n, lo + 1, mine, off, len(off))
        if kw["solver"] == 1:
            niter, iret = pdist.parcel_dcg_dia(*args, **common)
        elif kw["solver"] == 2:
            niter, iret = pdist.parcel_dbicgstab_dia(*args, **common)
        elif kw["solver"] == 3:
            niter, iret = pdist.parcel_dgmres_dia(*args, GMRES_m=kw["GMRES_m"], GMRES_GSflag=1, **common)
        else:
            niter, iret = pdist.parcel_dcagmres_dia(*args, CAGMRES_sstep=kw["CAGMRES_sstep"],
                                                    CAGMRES_tstep=kw["CAGMRES_tstep"],
                                                    CAGMRES_basis=kw["CAGMRES_basis"],
                                                    CAGMRES_QRflag=kw["CAGMRES_QRflag"], **common)
        q.put((rank, niter, iret, hist[:niter].copy(), x.numpy(), 0))
        dist.destroy_process_group()
    except Exception:  # pragma: no cover - reported to the parent
        import traceback
        q.put((rank, "error", traceback.format_exc(), None, None, None))


@pytest.mark.parametrize("kind", ["dia-cg", "dia-bicgstab", "dia-gmres", "dia-cagmres-4-2-1-5"])
def test_distributed_dia_rows_reproduce_the_crs_solve(kind):
    """Each process passes its rows of a DIA matrix (the diagonals in reverse offset order);
    the global columns (row + offset) reach the neighbouring process's rows through the halo
    exchange.  The histories equal the oracle's CRS solve of the same matrix as in the CRS
    tests (CA-GMRES at its own criteria)."""
    import cagmres
    import oracle
    world, nblocks = 2, 4
    A, b, kw = _problem(kind[4:])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dia_worker, args=(r, world, port, kind, nblocks, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
    for o in out:
        assert o[1] != "error", o[2]
    x = np.concatenate([o[4] for o in out])
    if kw["solver"] == 4:
        xo, ho, no, io = cagmres.pcagmres(A, b, s=kw["CAGMRES_sstep"], t=kw["CAGMRES_tstep"],
                                          basis=kw["CAGMRES_basis"], qrflag=kw["CAGMRES_QRflag"],
                                          itrmax=kw["itrmax"], rtolmax=kw["rtolmax"], ipreflag=2, ILU_method=0,
                                          precon_thblock=nblocks)
        for _, niter, iret, hist, _, _ in out:
            assert iret == io == 0 and abs(niter - no) <= 2
            k = min(niter, no)
            m = ho[:k] > 1e-8
            assert np.max(np.abs(hist[:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6
        assert oracle.true_relres(A, b, x) < 1e-9
        return
    okw = {k: v for k, v in kw.items() if not k.startswith("CAGMRES")}
    xo, ho, no, io = oracle.solve(A, b, ipreflag=2, ILU_method=0, precon_thblock=nblocks, **okw)
    for _, niter, iret, hist, _, _ in out:
        assert (niter, iret) == (no, io)
        m = ho[:niter] > 1e-8 * ho[0]
        assert np.max(np.abs(hist[m] - ho[:niter][m]) / ho[:niter][m]) < 1e-8
    assert np.max(np.abs(x - xo)) <= 1e-8 * np.max(np.abs(xo))


def test_dia_rows_global_columns_and_edges():
    """Row istart + k - 1 couples column row + offset; zero entries and columns outside
    1..gn are left out, each row's columns ascending; a repeated offset is refused."""
    from parcel_b import dist as pdist
    n, gn, istart = 3, 6, 3                        # rows 3, 4, 5 of 6
    off = np.array([2, -3, 0], np.int32)
    dia = np.array([[1.0, 2.0, 3.0],               # offset 2: columns 5, 6, 7 (7 is outside)
                    [4.0, 0.0, 6.0],               # offset -3: columns 0 (outside), 1 (zero), 2
                    [7.0, 8.0, 9.0]]).ravel()      # offset 0
    rp, col, val = pdist.dia_rows(n, gn, istart, dia, off, 3)
    assert rp.tolist() == [1, 3, 5, 7]
    assert col.tolist() == [3, 5, 4, 6, 2, 5]
    assert val.tolist() == [7.0, 1.0, 8.0, 2.0, 6.0, 9.0]
    with pytest.raises(ValueError):
        pdist.dia_rows(n, gn, istart, dia, np.array([0, 1, 0], np.int32), 3)
