"""Additive Schwarz with overlap over processes (parcel_b/schwarz.py) on CPU processes over gloo.

Two and three processes split the rows of a matrix contiguously; each builds the overlapped
additive Schwarz preconditioner of its rows (every block extended by addL rows on both
sides, into the neighbouring block or process; D-ILU on every region) with the local
block-Jacobi operator of the expanded matrix from the oracle.  Checked against the oracle's
global restatement (oracle/schwarz.py):
  * the application, for BASIC, RESTRICT, INTERPOLATE and NONE, ILUD and MLUD, to 1e-12
    relative (a row is covered by at most two regions, so the sums agree to rounding);
  * CG, BiCGStab, GMRES and CA-GMRES through it: the same iteration counts and histories
    (1e-8 relative while the residual is above 1e-8 of its start) as the same recurrences on
    one process with the oracle's global preconditioner;
  * the reference's fallbacks: block Jacobi on one process, and for every process when a
    block is shorter than 2 addL rows."""
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


def _matrix(kind):
    from parcel_b import problems
    if kind == "cg":
        A, b, _ = problems.poisson3d_reference(10, 10, 12)
        return A, b
    A = problems.convdiff3d_upwind(12)
    return A, problems.rhs_normal(A.n, 3)


def oracle_block_precon(n, rowptr, col, val, starts, options):
    """Local block-Jacobi D-ILU of an expanded matrix with explicit blocks, from the oracle."""
    import torch

    import oracle
    from parcel_b.problems import CRS
    M = oracle.Precon(oracle.Matrix(CRS(n=int(n), rowptr=np.asarray(rowptr, np.int32),
                                        col=np.asarray(col, np.int32), val=np.asarray(val, np.float64))),
                      ipreflag=2, ILU_method=int(options["ILU_method"]), blocks=np.asarray(starts, np.int64))

    class P:
        def precon(self, r, z):
            z.copy_(torch.from_numpy(np.asarray(M(r.numpy().copy()), dtype=np.float64)))
    return P()


class ScipySpmv:
    def __init__(self, lay, val):
        import scipy.sparse as sp
        import torch
        self.torch = torch
        self.A = sp.csr_matrix((val, lay.local_col.astype(np.int64) - 1, lay.rowptr.astype(np.int64) - 1),
                               shape=(lay.n, lay.n_ext))

    def spmv(self, x_ext, y):
        y.copy_(self.torch.from_numpy(self.A @ x_ext.numpy()))


SOLVER = {"cg": 1, "bicgstab": 2, "gmres": 3, "cagmres": 4}   # CA-GMRES: s = 4, t = 1, Cholesky QR


def _split(n, world):
    per = n // world
    return [(r * per, per if r < world - 1 else n - per * (world - 1)) for r in range(world)]


def _worker(rank, world, port, kind, nb, addL, iflag, ilu, solve, q):
    try:
        sys.path[:0] = [os.path.join(ROOT, "parcel-legacy_b200"), os.path.join(ROOT, "oracle")]
        import torch
        import torch.distributed as dist

        from parcel_b import dist as pdist
        from parcel_b.schwarz import Schwarz
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        A, b = _matrix(kind)
        lo, n = _split(A.n, world)[rank]
        rp = A.rowptr[lo:lo + n + 1] - A.rowptr[lo] + 1
        k0, k1 = A.rowptr[lo] - 1, A.rowptr[lo + n] - 1
        col, val = A.col[k0:k1], A.val[k0:k1]
        lay = pdist.Layout(n, A.n, lo + 1, rp, col)
        opts = dict(ILU_method=ilu)
        P = Schwarz(lay, rp, col, val, nb, addL, iflag, ilu, oracle_block_precon, opts)
        out = {"bj": P.bj}
        r = torch.from_numpy(np.random.default_rng(9).standard_normal(A.n)[lo:lo + n].copy())
        z = torch.zeros(n, dtype=torch.float64)
        P.precon(r, z)
        out["z"] = z.numpy()
        if solve:
            x = torch.zeros(n, dtype=torch.float64)
            be = pdist._Composed(ScipySpmv(lay, val), P)
            kw = dict(solver=SOLVER[kind], itrmax=400, rtolmax=1e-10, GMRES_m=10, GMRES_GSflag=1)
            niter, iret, hist = pdist.solve(lay, val, torch.from_numpy(b[lo:lo + n].copy()), x, backend=be, **kw)
            out.update(niter=niter, iret=iret, hist=hist, x=x.numpy())
        q.put((rank, out))
        dist.destroy_process_group()
    except Exception:
        import traceback
        q.put((rank, {"error": traceback.format_exc()}))


def _run(world, kind, nb, addL, iflag, ilu, solve=False):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, nb, addL, iflag, ilu, solve, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
    for _, o in out:
        assert "error" not in o, o.get("error")
    return [o for _, o in out]


@pytest.mark.parametrize("iflag", [1, 2, 3, 4], ids=["basic", "restrict", "interpolate", "none"])
@pytest.mark.parametrize("world,nb,ilu", [(2, 2, 1), (3, 2, 2)])
def test_distributed_schwarz_application_matches_oracle(iflag, world, nb, ilu):
    import schwarz
    A, _ = _matrix("gmres")
    addL = 40
    out = _run(world, "gmres", nb, addL, iflag, ilu)
    assert not any(o["bj"] for o in out)
    z = np.concatenate([o["z"] for o in out])
    r = np.random.default_rng(9).standard_normal(A.n)
    want = schwarz.apply(A, _split(A.n, world), nb, addL, iflag, r, ILU_method=ilu)
    assert np.max(np.abs(z - want)) <= 1e-12 * np.max(np.abs(want))
    # the overlap changes the preconditioner: not block Jacobi
    bj = schwarz.apply(A, _split(A.n, world), nb, 0, iflag, r, ILU_method=ilu)
    assert np.max(np.abs(want - bj)) > 1e-6 * np.max(np.abs(bj))


def test_short_blocks_fall_back_to_block_jacobi():
    import schwarz
    A, _ = _matrix("gmres")
    world, nb, addL = 2, 4, 400                      # blocks of 216 rows < 2 x 400
    out = _run(world, "gmres", nb, addL, 1, 1)
    assert all(o["bj"] for o in out)
    z = np.concatenate([o["z"] for o in out])
    r = np.random.default_rng(9).standard_normal(A.n)
    want = schwarz.apply(A, _split(A.n, world), nb, addL, 1, r)
    assert schwarz.falls_back(_split(A.n, world), nb, addL)
    assert np.max(np.abs(z - want)) <= 1e-12 * np.max(np.abs(want))


class _GlobalSchwarz:
    """One-process backend: the product and the oracle's global Schwarz preconditioner."""

    def __init__(self, A, ranges, nb, addL, iflag, ilu):
        import scipy.sparse as sp
        import torch
        self.torch = torch
        self.S = sp.csr_matrix((A.val, A.col - 1, A.rowptr - 1), shape=(A.n, A.n))
        self.args = (A, ranges, nb, addL, iflag)
        self.ilu = ilu

    def spmv(self, x_ext, y):
        y.copy_(self.torch.from_numpy(self.S @ x_ext.numpy()))

    def precon(self, r, z):
        import schwarz
        A, ranges, nb, addL, iflag = self.args
        z.copy_(self.torch.from_numpy(schwarz.apply(A, ranges, nb, addL, iflag, r.numpy(), ILU_method=self.ilu)))


@pytest.mark.parametrize("kind,world,iflag", [("cg", 2, 1), ("gmres", 3, 2), ("gmres", 2, 3), ("bicgstab", 2, 4),
                                               ("cagmres", 3, 1)])
def test_distributed_schwarz_solves_reproduce_the_global_recurrences(kind, world, iflag):
    import torch
    import torch.distributed as dist

    from parcel_b import dist as pdist
    A, b = _matrix(kind)
    nb, addL = 2, 30
    out = _run(world, kind, nb, addL, iflag, 1, solve=True)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1)
    try:
        lay = pdist.Layout(A.n, A.n, 1, A.rowptr, A.col)
        x = torch.zeros(A.n, dtype=torch.float64)
        be = _GlobalSchwarz(A, _split(A.n, world), nb, addL, iflag, 1)
        kw = dict(solver=SOLVER[kind], itrmax=400, rtolmax=1e-10, GMRES_m=10, GMRES_GSflag=1)
        no, io, ho = pdist.solve(lay, A.val, torch.from_numpy(b.copy()), x, backend=be, **kw)
    finally:
        dist.destroy_process_group()
    assert io == 0
    for o in out:
        assert (o["niter"], o["iret"]) == (no, io)
        m = ho > 1e-8 * ho[0]
        assert np.max(np.abs(o["hist"][m] - ho[m]) / ho[m]) < 1e-8
    xg = np.concatenate([o["x"] for o in out])
    assert np.max(np.abs(xg - x.numpy())) <= 1e-8 * np.max(np.abs(x.numpy()))
