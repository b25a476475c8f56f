"""The DDM stencil format on the GPU (parcel_b_solve_ddm, parcel_b_ddsolve_ddm and the
parcel_d*_ddm shims) against the oracle.

  * CG / BiCGStab / GMRES with block-Jacobi D-ILU on x, y and z slabs (the CPU build's
    boxes, uneven splits) and on the CUDA build's 4^3 boxes, and with point Jacobi and no
    preconditioner: the oracle's solve of the same global system (oracle/ddm.py) gives
    iterations +-2, histories within 1e-6 relative above 1e-8 of the start (BiCGStab: above
    1e-6 of the start; its recurrences amplify the different summation order of the dot
    products as the residual falls, to about 1e-4 relative at 1e-8 on the 4^3 boxes), x to
    1e-8; the margin of x is left as it was;
  * the double-double CG through the DDM box equals the oracle's dd CG on the renumbered
    system bit for bit (history, x_hi, x_lo);
  * the reference's stored CUDA-build DDM output (template_gpu/STDOUT_run_ddm: 160^3 with
    4^3 boxes, 345 CG iterations) through parcel_dcg_ddm_gpu_c_ with device arrays, history
    within 1e-6 relative;
  * the DDM path over processes with the GPU backend, in a one-process NCCL group;
  * what is not provided is refused with PARCEL_B_E_UNSUPPORTED.
"""
import ctypes as C
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

import ddm as oddm
import oracle
from conftest import golden
from parcel_b import _lib, ddm
from parcel_b.problems import CRS

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GN = (24, 20, 16)


def _oracle(p, boxes_of, **kw):
    G = oddm.global_system([p], (1, 1, 1), boxes_of)
    A = CRS(n=G["n"], rowptr=G["rowptr"], col=G["col"], val=G["val"])
    return G, oracle.solve(A, G["b"], blocks=G["starts"], **kw)


BOXES = [
    ("x-slabs-5", dict(boxes=ddm.BOXES_THREADS, div_direc_th=1, precon_thblock=5),
     lambda n: oddm.thread_boxes(n, 1, 5)),
    ("y-slabs-3", dict(boxes=ddm.BOXES_THREADS, div_direc_th=2, precon_thblock=3),
     lambda n: oddm.thread_boxes(n, 2, 3)),
    ("z-slabs-4", dict(boxes=ddm.BOXES_THREADS, div_direc_th=3, precon_thblock=4),
     lambda n: oddm.thread_boxes(n, 3, 4)),
    ("cubes", dict(boxes=ddm.BOXES_CUBES), oddm.cube_boxes),
]


@pytest.mark.parametrize("solver", [1, 2, 3], ids=["cg", "bicgstab", "gmres"])
@pytest.mark.parametrize("name,opt,boxes_of", BOXES, ids=[b[0] for b in BOXES])
def test_ddm_solve_matches_oracle(solver, name, opt, boxes_of):
    p = oddm.poisson3d_ddm(GN, (1, 1, 1), 0)
    kw = dict(solver=solver, ipreflag=2, itrmax=600, rtolmax=1e-10, GMRES_m=12, GMRES_GSflag=1)
    G, (xo, ho, no, io) = _oracle(p, boxes_of, ILU_method=1, **kw)
    x0 = np.zeros(p["m"])
    margin = np.ones(p["m"], bool)
    margin[G["padded"]] = False
    x0[margin] = 7.0                        # the margin must come back untouched
    g = ddm.solve(p["val"], p["offset"], p["offset_dim"], p["n"], p["b"], x0, **opt, **kw)
    assert g["iret"] == io == 0 and abs(g["niter"] - no) <= 2, (g["niter"], no)
    k = min(g["niter"], no)
    m = ho[:k] > (1e-6 if solver == 2 else 1e-8) * ho[0]
    assert np.max(np.abs(g["reshistory"][:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6
    x = g["x"]
    assert np.max(np.abs(x[G["padded"]] - xo)) <= 1e-8 * np.max(np.abs(xo))
    assert np.all(x[margin] == 7.0)
    assert g["stats"]["ilu_nblocks"] == len(boxes_of(p["n"]))


def test_ddm_solve_into_out_in_place():
    """out= holds the initial guess and receives x in place (page-locked host memory and a
    device tensor); the same result as the x0 form, bit for bit."""
    import torch
    p = oddm.poisson3d_ddm(GN, (1, 1, 1), 0)
    kw = dict(solver=1, ipreflag=2, itrmax=600, rtolmax=1e-10, boxes=ddm.BOXES_CUBES)
    x0 = np.zeros(p["m"])
    x0[0] = 3.0                              # a margin cell: must come back untouched
    g = ddm.solve(p["val"], p["offset"], p["offset_dim"], p["n"], p["b"], x0, **kw)
    h = torch.from_numpy(x0.copy()).pin_memory().numpy()
    r = ddm.solve(p["val"], p["offset"], p["offset_dim"], p["n"], p["b"], out=h, **kw)
    assert r["x"] is h and np.array_equal(h, g["x"]) and h[0] == 3.0
    assert r["niter"] == g["niter"] and np.array_equal(r["reshistory"], g["reshistory"])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d = t(x0)
    r = ddm.solve(t(p["val"]), t(p["offset"]), t(p["offset_dim"]), p["n"], t(p["b"]), out=d, **kw)
    assert np.array_equal(d.cpu().numpy(), g["x"])


@pytest.mark.parametrize("ipreflag", [0, 1])
def test_ddm_point_jacobi_and_none_match_oracle(ipreflag):
    p = oddm.poisson3d_ddm(GN, (1, 1, 1), 0)
    kw = dict(solver=1, ipreflag=ipreflag, itrmax=800, rtolmax=1e-9)
    G, (xo, ho, no, io) = _oracle(p, oddm.cube_boxes, **kw)
    g = ddm.solve(p["val"], p["offset"], p["offset_dim"], p["n"], p["b"], **kw)
    assert g["iret"] == io == 0 and abs(g["niter"] - no) <= 2
    k = min(g["niter"], no)
    m = ho[:k] > 1e-8 * ho[0]
    assert np.max(np.abs(g["reshistory"][:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6


def test_ddm_ddcg_matches_oracle_bit_for_bit():
    p = oddm.poisson3d_ddm((20, 16, 12), (1, 1, 1), 0)
    kw = dict(ipreflag=2, itrmax=400, rtolmax=1e-12)
    g = ddm.ddsolve(p["val"], p["offset"], p["offset_dim"], p["n"], p["b"], div_direc_th=2, precon_thblock=3,
                    **kw)
    G = oddm.global_system([p], (1, 1, 1), lambda n: oddm.thread_boxes(n, 2, 3))
    A = CRS(n=G["n"], rowptr=G["rowptr"], col=G["col"], val=G["val"])
    xh, xl, h, niter, iret = oracle.ddcg(A, G["b"], ILU_method=1, blocks=G["starts"], **kw)
    assert g["iret"] == iret == 0 and g["niter"] == niter
    assert np.array_equal(g["reshistory"], h)
    assert np.array_equal(g["x_hi"][G["padded"]], xh) and np.array_equal(g["x_lo"][G["padded"]], xl)


def test_gpu_ddm_template_through_the_cuda_build_shim():
    import torch
    fx = golden()["gpu_ddm_cg_cubes"]
    p = oddm.poisson3d_ddm((160, 160, 160), (1, 1, 1), 0)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    x, b, val, off = dev(np.zeros(p["m"])), dev(p["b"]), dev(p["val"]), dev(p["offset"])
    handle = lambda t: C.c_void_p(t.data_ptr())
    hx, hb, hv, ho = handle(x), handle(b), handle(val), handle(off)
    i = lambda v: C.byref(C.c_int(v))
    hist = np.zeros(2000)
    niter, iret = C.c_int(2000), C.c_int(0)
    odim = np.ascontiguousarray(p["offset_dim"], np.int32)
    n_grids, npe = np.array(p["n"], np.int32), np.ones(3, np.int32)
    nbr = np.zeros(1, np.int32)
    L = _lib.load()
    L.parcel_dcg_ddm_gpu_c_(i(0), C.byref(hx), C.byref(hb), C.byref(C.c_int32(p["m"])), i(7), C.byref(ho),
                            C.byref(hv), i(0), nbr.ctypes.data_as(_lib.IP), i(1), i(3),
                            npe.ctypes.data_as(_lib.IP), n_grids.ctypes.data_as(_lib.IP),
                            odim.ctypes.data_as(_lib.IP), i(1), i(2), i(2), i(1), C.byref(niter),
                            C.byref(C.c_double(1e-9)), hist.ctypes.data_as(C.c_void_p), i(0), i(-1), i(1), i(-1),
                            i(2000), C.byref(iret))
    g = np.array(fx["history"])
    assert iret.value == 0 and niter.value == len(g) == 345
    rel = np.abs(hist[:niter.value] - g) / g
    assert rel.max() <= 1e-6, rel.max()
    err = np.abs(x.cpu().numpy() - p["x_exact"]).max() / np.abs(p["x_exact"]).max()
    assert err < 1e-6


def test_ddm_refuses_what_is_not_provided():
    p = oddm.poisson3d_ddm((8, 8, 8), (1, 1, 1), 0)
    args = (p["val"], p["offset"], p["offset_dim"], p["n"], p["b"])
    for kw in (dict(ipreflag=3), dict(ipreflag=4), dict(ipreflag=2, independ_nvec=1),
               dict(ipreflag=2, div_direc_th=0)):
        with pytest.raises(RuntimeError):
            ddm.solve(*args, solver=1, **kw)
    # the C-callable form with a box split over two processes
    i = lambda v: C.byref(C.c_int(v))
    odim = np.ascontiguousarray(p["offset_dim"], np.int32)
    n_grids, npe, nbr = np.array(p["n"], np.int32), np.array([1, 2, 1], np.int32), np.zeros(1, np.int32)
    x, hist = np.zeros(p["m"]), np.zeros(10)
    niter, iret = C.c_int(10), C.c_int(0)
    _lib.load().parcel_dcg_ddm_c_(i(0), x.ctypes.data_as(C.c_void_p), p["b"].ctypes.data_as(C.c_void_p),
                                  C.byref(C.c_int32(p["m"])), i(7), p["offset"].ctypes.data_as(_lib.I32P),
                                  p["val"].ctypes.data_as(C.c_void_p), i(0), nbr.ctypes.data_as(_lib.IP), i(1),
                                  i(3), npe.ctypes.data_as(_lib.IP), n_grids.ctypes.data_as(_lib.IP),
                                  odim.ctypes.data_as(_lib.IP), i(1), i(2), i(2), i(1), C.byref(niter),
                                  C.byref(C.c_double(1e-9)), hist.ctypes.data_as(C.c_void_p), i(0), i(4), i(1),
                                  i(-1), i(2000), C.byref(iret))
    assert iret.value == -5 and niter.value == 0   # PARCEL_B_E_UNSUPPORTED


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _child(port, q):
    try:
        sys.path[:0] = [os.path.join(ROOT, "parcel-legacy_b200"), os.path.join(ROOT, "oracle")]
        import torch
        import torch.distributed as dist

        import ddm as od
        from parcel_b import ddm as pd
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
        p = od.poisson3d_ddm(GN, (1, 1, 1), 0)
        x = torch.zeros(p["m"], dtype=torch.float64, device="cuda")
        b = torch.from_numpy(p["b"]).cuda()
        hist = np.zeros(600)
        niter, iret = pd.parcel_dcg_ddm(x, b, p["m"], 7, p["offset"], p["val"], 0, np.zeros(0, np.int32), 1, 3,
                                        np.ones(3, np.int32), np.array(p["n"]), p["offset_dim"], 1, 2, 2, 1, 600,
                                        1e-10, hist, 0, 5, 1, -1, 0)
        q.put((niter, iret, hist[:niter].copy(), x.cpu().numpy()))
        dist.destroy_process_group()
    except Exception:
        import traceback
        q.put(("error", traceback.format_exc(), None, None))


def test_ddm_over_processes_on_the_gpu_backend():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pr = ctx.Process(target=_child, args=(_free_port(), q))
    pr.start()
    niter, iret, hist, x = q.get(timeout=600)
    pr.join(timeout=60)
    assert niter != "error", iret
    p = oddm.poisson3d_ddm(GN, (1, 1, 1), 0)
    G, (xo, ho, no, io) = _oracle(p, lambda n: oddm.thread_boxes(n, 1, 5), solver=1, ipreflag=2, ILU_method=1,
                                  itrmax=600, rtolmax=1e-10)
    assert iret == io and abs(niter - no) <= 2
    k = min(niter, no)
    m = ho[:k] > 1e-8 * ho[0]
    assert np.max(np.abs(hist[:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6
    assert np.max(np.abs(x[G["padded"]] - xo)) <= 1e-8 * np.max(np.abs(xo))


GENERAL = [
    ("star13-margin2-xslabs", (12, 10, 8), 2, "star", dict(boxes=ddm.BOXES_THREADS, div_direc_th=1, precon_thblock=3),
     lambda n: oddm.thread_boxes(n, 1, 3)),
    ("star13-margin2-cubes", (12, 10, 8), 2, "star", dict(boxes=ddm.BOXES_CUBES), oddm.cube_boxes),
    ("box27-zslabs", (10, 9, 8), 1, "box", dict(boxes=ddm.BOXES_THREADS, div_direc_th=3, precon_thblock=2),
     lambda n: oddm.thread_boxes(n, 3, 2)),
    ("2d-box9-yslabs", (40, 30), 1, "box", dict(boxes=ddm.BOXES_THREADS, div_direc_th=2, precon_thblock=4),
     lambda n: oddm.thread_boxes(n, 2, 4)),
    ("2d-box9-cubes", (40, 30), 1, "box", dict(boxes=ddm.BOXES_CUBES), oddm.cube_boxes),
]


@pytest.mark.parametrize("solver", [2, 3], ids=["bicgstab", "gmres"])
@pytest.mark.parametrize("name,n,margin,kind,opt,boxes_of", GENERAL, ids=[g[0] for g in GENERAL])
def test_ddm_general_stencils_match_oracle(solver, name, n, margin, kind, opt, boxes_of):
    """Boxes the reference's example does not make: a 13-point star reaching two cells (margin
    2), the 27-point box (13 couplings per row and sweep, the general sweep) and a 2D box,
    with random nonsymmetric couplings; against the oracle's solve of the renumbered system
    with the boxes as blocks (every coupling that leaves a box dropped)."""
    import ddm_cases
    pts = ddm_cases.star(len(n), 2) if kind == "star" else ddm_cases.box(len(n))
    p = ddm_cases.stencil_box(n, margin, pts, seed=11)
    kw = dict(solver=solver, ipreflag=2, itrmax=800, rtolmax=1e-10, GMRES_m=15, GMRES_GSflag=1)
    G, (xo, ho, no, io) = _oracle(p, boxes_of, ILU_method=1, **kw)
    g = ddm.solve(p["val"], p["offset"], p["offset_dim"], n, p["b"], margin=margin, **opt, **kw)
    assert g["iret"] == io == 0 and abs(g["niter"] - no) <= 2, (g["niter"], no)
    k = min(g["niter"], no)
    m = ho[:k] > (1e-6 if solver == 2 else 1e-8) * ho[0]
    assert np.max(np.abs(g["reshistory"][:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6
    assert np.max(np.abs(g["x"][G["padded"]] - xo)) <= 1e-7 * np.max(np.abs(xo))
    assert g["stats"]["ilu_nblocks"] == len(boxes_of(p["n"]))
