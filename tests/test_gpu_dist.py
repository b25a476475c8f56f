"""The GPU backend of the row-distributed solve: parcel_b_local_* through the C-ABI.

  * the local operator of one process's rows (owned columns plus halo columns) against
    numpy (product, 1e-13 relative) and against the oracle's block-Jacobi ILU(0) on the
    owned-owned submatrix (preconditioner, 1e-12 relative);
  * the distributed recurrences with the GPU backend in a one-process NCCL group against
    the oracle (iterations +-2, histories 1e-6 relative above 1e-8 of the start).
Several processes on one GPU are not run: their NCCL transfers wait on one another, and
nothing makes two processes' kernels run at the same time on one GPU; the multi-process
logic is covered on CPU processes in tests/test_dist.py."""
import ctypes as C
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

import oracle
from parcel_b import _lib, api, problems

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _local_rows(A, lo, hi):
    """Rows lo..hi-1 of A with local column ids: owned 1..n, halo n+1.. (ascending global)."""
    rp = A.rowptr[lo:hi + 1] - A.rowptr[lo] + 1
    k0, k1 = A.rowptr[lo] - 1, A.rowptr[hi] - 1
    col = A.col[k0:k1].astype(np.int64)
    own = (col >= lo + 1) & (col <= hi)
    ghost = np.unique(col[~own])
    local = np.where(own, col - lo, hi - lo + 1 + np.searchsorted(ghost, col))
    return rp.astype(np.int32), local.astype(np.int32), A.val[k0:k1].copy(), ghost


def test_local_operator_matches_numpy_and_oracle():
    import scipy.sparse as sp
    import torch
    A = problems.convdiff3d_upwind(16)
    lo, hi = A.n // 4, 3 * A.n // 4                   # the middle half: halo rows on both sides
    rp, ci, va, ghost = _local_rows(A, lo, hi)
    n, n_ext = hi - lo, hi - lo + len(ghost)
    L = _lib.load()
    p = _lib.new_input(solver=3, ipreflag=2, ILU_method=0, precon_thblock=4)
    S = _lib.Crs(n, n, int(ci.shape[0]), 1, rp.ctypes.data, ci.ctypes.data, va.ctypes.data)
    h = C.c_void_p()
    assert L.parcel_b_local_create(C.byref(p), C.byref(S), n_ext, C.byref(h)) == 0, _lib.last_error()
    try:
        rng = np.random.default_rng(1)
        xe = rng.standard_normal(n_ext)
        y = torch.zeros(n, dtype=torch.float64, device="cuda")
        xd = torch.from_numpy(xe).cuda()
        assert L.parcel_b_local_spmv(h, xd.data_ptr(), y.data_ptr()) == 0, _lib.last_error()
        want = sp.csr_matrix((va, ci - 1, rp - 1), shape=(n, n_ext)) @ xe
        assert np.linalg.norm(y.cpu().numpy() - want) <= 1e-13 * np.linalg.norm(want)
        # preconditioner: the oracle's block Jacobi (4 blocks) on the owned-owned submatrix
        own = sp.csr_matrix((va, ci - 1, rp - 1), shape=(n, n_ext))[:, :n].tocsr()
        own.sort_indices()
        Aoo = problems.CRS(n=n, rowptr=(own.indptr + 1).astype(np.int32), col=(own.indices + 1).astype(np.int32),
                           val=own.data.copy())
        r = rng.standard_normal(n)
        z = torch.zeros(n, dtype=torch.float64, device="cuda")
        rd = torch.from_numpy(r).cuda()
        assert L.parcel_b_local_precon(h, rd.data_ptr(), z.data_ptr()) == 0, _lib.last_error()
        zo = oracle.precon_apply(Aoo, r, ipreflag=2, ILU_method=0, precon_thblock=4)
        assert np.linalg.norm(z.cpu().numpy() - zo) <= 1e-12 * np.linalg.norm(zo)
    finally:
        L.parcel_b_local_destroy(h)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _child(port, kind, q):
    try:
        sys.path[:0] = [os.path.join(ROOT, "parcel-legacy_b200"), os.path.join(ROOT, "oracle")]
        import torch
        import torch.distributed as dist

        from parcel_b import dist as pdist
        from parcel_b import problems as pr
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
        if kind == "cg":
            A, b, _ = pr.poisson3d_reference(24, 24, 24)
            kw = dict(solver=1, itrmax=500, rtolmax=1e-9, ipreflag=2, ILU_method=0, precon_thblock=4)
        else:
            A = pr.convdiff3d_upwind(24)
            b = pr.rhs_normal(A.n, 3)
            kw = dict(solver=3, itrmax=1000, rtolmax=1e-10, GMRES_m=20, GMRES_GSflag=1, ipreflag=2, ILU_method=0,
                      precon_thblock=4)
        lay = pdist.Layout(A.n, A.n, 1, A.rowptr, A.col)
        x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
        niter, iret, hist = pdist.solve(lay, A.val, torch.from_numpy(b).cuda(), x, **kw)
        q.put((niter, iret, hist, x.cpu().numpy()))
        dist.destroy_process_group()
    except Exception:
        import traceback
        q.put(("error", traceback.format_exc(), None, None))


@pytest.mark.parametrize("kind", ["cg", "gmres"])
def test_distributed_recurrences_on_the_gpu_backend(kind):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_child, args=(_free_port(), kind, q))
    p.start()
    niter, iret, hist, x = q.get(timeout=600)
    p.join(timeout=60)
    assert niter != "error", iret
    if kind == "cg":
        A, b, _ = problems.poisson3d_reference(24, 24, 24)
        kw = dict(solver=1, itrmax=500, rtolmax=1e-9)
    else:
        A = problems.convdiff3d_upwind(24)
        b = problems.rhs_normal(A.n, 3)
        kw = dict(solver=3, itrmax=1000, rtolmax=1e-10, GMRES_m=20, GMRES_GSflag=1)
    xo, ho, no, io = oracle.solve(A, b, ipreflag=2, ILU_method=0, precon_thblock=4, **kw)
    assert iret == io and abs(niter - no) <= 2, (niter, iret, no, io)
    k = min(niter, no)
    m = ho[:k] > 1e-8 * ho[0]
    assert np.max(np.abs(hist[:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6
    assert oracle.true_relres(A, b, x) < 10 * kw["rtolmax"]


@pytest.mark.parametrize("ilu", [1, 2])
def test_expanded_region_operator_matches_oracle(ilu):
    """The GPU side of the overlapped additive Schwarz (parcel_b/schwarz.py): the library's
    block-Jacobi D-ILU of an expanded matrix whose blocks are overlapping regions of A (rows
    repeated in each region that covers them), through dist.cuda_block_precon, against the
    oracle's block Jacobi with the same explicit blocks (1e-12 relative)."""
    import scipy.sparse as sp
    import torch

    from parcel_b import dist as pdist
    from parcel_b.problems import CRS
    A = problems.convdiff3d_upwind(14)
    S = sp.csr_matrix((A.val, A.col - 1, A.rowptr - 1), shape=(A.n, A.n))
    regions = [(0, 1000), (900, 2000), (1900, A.n)]
    subs = [S[a:b, a:b].tocsr() for a, b in regions]
    E = sp.block_diag(subs, format="csr")
    E.sort_indices()
    starts = [0]
    for a, b in regions:
        starts.append(starts[-1] + b - a)
    M = pdist.cuda_block_precon(E.shape[0], (E.indptr + 1).astype(np.int32), (E.indices + 1).astype(np.int32),
                                E.data.copy(), starts, dict(ipreflag=2, ILU_method=ilu))
    r = np.random.default_rng(7).standard_normal(E.shape[0])
    z = torch.zeros(E.shape[0], dtype=torch.float64, device="cuda")
    M.precon(torch.from_numpy(r).cuda(), z)
    Ec = CRS(n=E.shape[0], rowptr=(E.indptr + 1).astype(np.int32), col=(E.indices + 1).astype(np.int32),
             val=E.data.copy())
    want = oracle.precon_apply(Ec, r, ipreflag=2, ILU_method=ilu, blocks=starts)
    assert np.linalg.norm(z.cpu().numpy() - want) <= 1e-12 * np.linalg.norm(want)
