"""Benchmark: time to a 1e-10 true relative residual for PARCEL's drop-in GMRES path.

Workload (one "step" = one complete solve): 3D 7-point upwind convection-diffusion on a
128^3 grid (n = 2,097,152, nnz = 14,581,760, CRS int32), -Lap u + Pe v.grad u with
v = (1, 0.5, 0.25), Pe = 10, h = 1/129; b ~ N(0,1) (seed 2); x0 = 0; GMRES(30) with
modified Gram-Schmidt (the reference default) and block-Jacobi ILU(0) over 64
contiguous-row blocks; stop at relative residual 1e-10.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value : device time (CUDA events on the library stream) of the whole solve call
        (setup + iteration) through the GPU-build C-ABI (parcel_dgmres_gpu_c_) with the
        matrix and vectors already in HBM.
e2e   : the same solve through the CPU-build C-ABI (parcel_dgmres_c_) with host arrays,
        host<->device copies inside the timed region.
roofline : the CRS SpMV kernel (the metric's "SpMV HBM GB/s"), algorithmic bytes
        (8+4) nnz + 4 (n+1) + 8 n + 8 n per launch over its CUDA-event time.
--impl reference : the reference's CPU algorithm (the oracle port of KSP_pGMRES with
        block-Jacobi ILU(0)) on the host cores, same workload and metric.
With torchrun (N > 1) every rank solves its own copy of the problem on its GPU (replicas;
the solve is not split across GPUs), and the slowest rank's time is reported.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "parcel-legacy_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

N_GRID = 128
NBLOCKS = 64
GMRES_M = 30
RTOL = 1e-10
ITRMAX = 5000
SEED_B = 2
METRIC = "time-to-1e-10 true rel. residual (s) vs plain FP64 GPU path; SpMV HBM GB/s"
WORKLOAD = ("PGMRES(30) FP64, block-Jacobi ILU(0) 64 blocks, 3D 7-pt upwind convection-diffusion "
            "128^3 (Pe=10, v=(1,0.5,0.25)), b~N(0,1), tol 1e-10")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def config(world):
    """The workload description both arms print (the reference arm runs the same problem)."""
    return {"workload": WORKLOAD, "n": 2097152, "nnz": 14581760, "blocks": NBLOCKS, "restart": GMRES_M,
            "orthogonalization": "MGS", "l2": "inputs larger than L2 (217 MB matrix, 126 MB L2)",
            "parallelism": f"replicas x{world}"}


def problem():
    from parcel_b import problems
    A = problems.convdiff3d_upwind(N_GRID)
    b = problems.rhs_normal(A.n, SEED_B)
    return A, b


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def started(self, timeout: float = 5.0):
        """Waits for the first sample, so that nvidia-smi's own start-up (which competes
        for the host cores the set-up uses) lies before the timed region."""
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < timeout:
            if os.path.getsize(self.f.name) > 0:
                return
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [l.strip().split(", ") for l in open(self.f.name) if l.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        load = [s for s in sm if s > 300] or sm
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(rows)}


def reduce_max(values, dist=None, device=None):
    """Element-wise maximum of a list of floats over all ranks (the slowest rank's times);
    the values themselves on a single process."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def dist_setup(ngpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_ours(args):
    import torch
    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from parcel_b import _lib, api
    L = _lib.load()
    A, b = problem()
    dev = torch.device("cuda", local)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rp, ci, va, bd = t(A.rowptr), t(A.col), t(A.val), t(b)
    x = torch.zeros(A.n, dtype=torch.float64, device=dev)
    hist = np.zeros(ITRMAX)
    stream = torch.cuda.ExternalStream(L.parcel_b_get_stream(), device=dev)

    def solve_dev():
        x.zero_()
        torch.cuda.synchronize()
        return api.parcel_dgmres(x, bd, A.n, A.n, A.nnz, 1, va, rp, ci, 2, 0, 0, 1, ITRMAX, RTOL, hist,
                                 precon_thblock=NBLOCKS, GMRES_m=GMRES_M, GMRES_GSflag=1)

    # pinned host copies for the end-to-end arm
    hp = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_rp, h_ci, h_va, h_b = hp(A.rowptr), hp(A.col), hp(A.val), hp(b)
    h_x = torch.zeros(A.n, dtype=torch.float64).pin_memory().numpy()

    def solve_host():
        h_x[:] = 0.0
        return api.parcel_dgmres(h_x, h_b, A.n, A.n, A.nnz, 1, h_va, h_rp, h_ci, 2, 0, 0, 1, ITRMAX, RTOL,
                                 hist, precon_thblock=NBLOCKS, GMRES_m=GMRES_M, GMRES_GSflag=1)

    for _ in range(args.warmup):
        niter, iret = solve_dev()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.started()
    times, stats = [], []
    for _ in range(args.steps):
        x.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        niter, iret = api.parcel_dgmres(x, bd, A.n, A.n, A.nnz, 1, va, rp, ci, 2, 0, 0, 1, ITRMAX, RTOL, hist,
                                        precon_thblock=NBLOCKS, GMRES_m=GMRES_M, GMRES_GSflag=1)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
        stats.append(_lib.last_stats())
    torch.cuda.synchronize()
    clocks = clk.stop()
    step_s, tot = reduce_max([max(times), sum(times)], dist, dev)
    value = tot / args.steps
    relres = stats[-1]["true_relres"]

    # end-to-end: host arrays through the CPU-build ABI, copies inside the timed region
    solve_host()
    torch.cuda.synchronize()
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        n2, i2 = solve_host()
        e2e.append(time.perf_counter() - t0)
    h2d = A.rowptr.nbytes + A.col.nbytes + A.val.nbytes + 2 * A.n * 8
    d2h = A.n * 8 + ITRMAX * 8

    # kernel timing for the roofline (CUDA events on the library stream)
    ms_spmv, ms_pre = C.c_double(0), C.c_double(0)
    p = _lib.new_input(solver=3, ipreflag=2, ILU_method=0, precon_thblock=NBLOCKS, GMRES_m=GMRES_M)
    S = api.crs_struct(A, rp, ci, va)
    rc = L.parcel_b_bench_kernels(C.byref(p), C.byref(S), 50, C.byref(ms_spmv), C.byref(ms_pre))
    assert rc == 0, _lib.last_error()
    hbm, peak_kind = peaks()
    spmv_bytes = 12 * A.nnz + 4 * (A.n + 1) + 16 * A.n
    achieved = spmv_bytes / (ms_spmv.value * 1e-3) / 1e9
    # DRAM bytes (read + write) of one k_spmv_sell launch on this workload, from one
    # `ncu --set full --clock-control none -k regex:k_spmv_sell -s 1 -c 1` capture of
    # `bench.py --kernels-only`:
    # dram__bytes_read.sum 196.24 MB + dram__bytes_write.sum 5.30 MB (cold cache).
    spmv_traffic = 196.237568e6 + 5.297664e6
    # the step's dominant kernel: the block-Jacobi ILU(0) application (forward + backward
    # sweep), algorithmic bytes 12 nnz + 8 (n + 1) + 32 n (L and U values and columns, row
    # pointers, r read, z written twice); DRAM bytes of one k_ilu_sweep_grp launch from one
    # `ncu --set full --clock-control none -k regex:k_ilu_sweep_grp -s 3 -c 1` capture of
    # `bench.py --kernels-only --steps 5`: read 199.03 MB + write 23.18 MB.
    ilu_bytes = 12 * A.nnz + 8 * (A.n + 1) + 32 * A.n
    ilu_achieved = ilu_bytes / (ms_pre.value * 1e-3) / 1e9
    ilu_traffic = 199.030784e6 + 23.179264e6

    out = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config(world),
        "iterations": niter, "iret": iret, "true_relres": relres,
        "step_times_s": [round(t_, 6) for t_ in times],
        "setup_s": stats[-1]["setup_s"], "solve_s": stats[-1]["solve_s"],
        "e2e": {"value": sum(e2e) / len(e2e), "unit": "s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "kernel": "k_spmv_sell<double,double> (sliced-ELLPACK SpMV, level-major layout)",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "traffic": int(spmv_traffic), "algorithmic_bytes": int(spmv_bytes),
                     "us_per_launch": ms_spmv.value * 1e3},
        "roofline_dominant": {"bound": "hbm (the sweep is level-latency bound: 2 x 256 dependent levels per block)",
                              "kernel": "k_ilu_sweep_grp<double> (block-Jacobi ILU(0) apply, 64 CTAs)",
                              "achieved": ilu_achieved, "peak": hbm, "unit": "GB/s", "frac": ilu_achieved / hbm,
                              "peak_kind": peak_kind, "traffic": int(ilu_traffic),
                              "algorithmic_bytes": int(ilu_bytes), "us_per_launch": ms_pre.value * 1e3,
                              "launches_per_step": niter - (-niter // GMRES_M)},
        "kernels_us": {"spmv": ms_spmv.value * 1e3, "bj_ilu0_apply": ms_pre.value * 1e3},
        "clocks": clocks,
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
    }
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(A, b)
    if world == 1 and args.target_rhs > 0:   # one process only: the other ranks would wait on a barrier
        out["target"] = target_summary(args)
    if world == 1 and not args.no_configs:
        out["configs_gpu"] = configs_summary()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def target_summary(args):
    """The learned + mixed-precision target on its own workload (256^3 variable-coefficient
    diffusion), with a reduced number of right-hand sides: seconds per right-hand side of
    the plain FP64 path, the mixed-precision path without the stage, the coarse stage
    without and with the network, and the coarse stage at 8 steps without the network."""
    v = vardiff_compare(args.grid, args.coarsen, args.restart, args.target_rhs, args.target_rhs,
                        args.target_train_rhs, args.target_train_steps, k=args.coarse_steps)
    arms = ("plain_fp64", "mixed_no_stage", "mixed_coarse", "learned", "mixed_coarse_k8")
    return {"workload": v["config"]["workload"], "rhs": args.target_rhs,
            "s_per_rhs": {a: v[a]["s_per_rhs_amortised"] for a in arms},
            "speedup": v["speedup_vs_plain_fp64"],
            "network_gain": v["network_gain"],
            "iterations": {a: v[a]["iterations"] for a in arms},
            "true_relres_max": {a: v[a]["true_relres_max"] for a in arms},
            "training": v["training"]}


def configs_summary():
    """GPU time, iterations and true residual of the other configurations and of the
    double-double solvers, each one warm-up and two timed solves with the arrays in HBM (CUDA
    events on the library stream), so that the default line carries them too; their full
    lines (e2e, CPU baselines, rooflines) come from --workload."""
    import torch
    from parcel_b import _lib, api, problems
    import oracle
    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.ExternalStream(L.parcel_b_get_stream(), device=dev)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    def timed(fn, reps=2):
        fn()
        ts, out = [], None
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return min(ts), out

    out = {}
    for name in ("poisson2d256", "aniso192", "banded4m"):
        c = _cfg(name)
        A, b = c["A"], c["b"]
        rp, ci, va, bd = t(A.rowptr), t(A.col), t(A.val), t(b)
        sec, r = timed(lambda: api.solve(A, bd, rowptr=rp, col=ci, val=va, **c["opts"]))
        out[name] = {"s": sec, "iterations": r["niter"], "iret": r["iret"],
                     "true_relres": oracle.true_relres(A, b, r["x"].cpu().numpy())}
        del rp, ci, va, bd
    A, b, xe = problems.poisson3d_reference(160, 160, 160)
    rp, ci, va, bd = t(A.rowptr), t(A.col), t(A.val), t(b)
    sec, r = timed(lambda: api.ddcg(A, bd, rowptr=rp, col=ci, val=va, itrmax=2000, rtolmax=1e-9, ipreflag=2,
                                    ILU_method=1, precon_thblock=80))
    x = r["x_hi"].cpu().numpy() + r["x_lo"].cpu().numpy()
    out["ddcg160"] = {"s": sec, "iterations": r["niter"], "iret": r["iret"],
                      "max_abs_error": float(np.abs(x - xe).max())}
    A, b = problem()
    rp, ci, va, bd = t(A.rowptr), t(A.col), t(A.val), t(b)
    sec, r = timed(lambda: api.ddgmres(A, bd, rowptr=rp, col=ci, val=va, itrmax=3000, rtolmax=1e-10, ipreflag=2,
                                       ILU_method=1, precon_thblock=NBLOCKS, GMRES_m=GMRES_M, GMRES_GSflag=1), reps=1)
    x = r["x_hi"].cpu().numpy() + r["x_lo"].cpu().numpy()
    out["ddgmres128"] = {"s": sec, "iterations": r["niter"], "iret": r["iret"],
                         "true_relres": oracle.true_relres(A, b, x)}
    import ddm as oddm
    from parcel_b import ddm
    p = oddm.poisson3d_ddm((160, 160, 160), (1, 1, 1), 0)
    val, off, bd = t(p["val"]), t(p["offset"]), t(p["b"])
    sec, r = timed(lambda: ddm.solve(val, off, p["offset_dim"], p["n"], bd, boxes=ddm.BOXES_CUBES, solver=1,
                                     ipreflag=2, itrmax=2000, rtolmax=1e-9))
    x = r["x"].cpu().numpy()
    out["ddm160"] = {"s": sec, "iterations": r["niter"], "iret": r["iret"], "template_iterations": 345,
                     "max_rel_error": float(np.abs(x - p["x_exact"]).max() / np.abs(p["x_exact"]).max())}
    return out


def cpu_baseline(A, b):
    import oracle
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    t0 = time.perf_counter()
    x, h, niter, iret = oracle.solve(A, b, solver=3, ipreflag=2, ILU_method=0, precon_thblock=NBLOCKS,
                                     itrmax=ITRMAX, rtolmax=RTOL, GMRES_m=GMRES_M, GMRES_GSflag=1)
    dt = time.perf_counter() - t0
    return {"value": dt, "unit": "s", "cores": cores, "kind": "port",
            "sample": f"one full oracle solve of the same workload ({niter} GMRES iterations, iret {iret})"}


def run_reference(args):
    rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import oracle
    A, b = problem()
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    M = oracle.Matrix(A)
    times = []
    niter = 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        x, h, niter, iret = oracle.solve(M, b, solver=3, ipreflag=2, ILU_method=0, precon_thblock=NBLOCKS,
                                         itrmax=ITRMAX, rtolmax=RTOL, GMRES_m=GMRES_M, GMRES_GSflag=1)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    value = sum(times) / len(times)
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": config(world),
           "iterations": niter,
           "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port",
                            "sample": "full solves of the same workload by the C++/OpenMP restatement of "
                                      "KSP_pGMRES + block-Jacobi ILU(0) (the reference's Fortran cannot be "
                                      "built here)"},
           "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_reference_dd(args):
    """Reference arm of the dd workloads: the oracle's restatement of ddKSP_pCG (ddcg160) or
    ddKSP_pGMRES (ddgmres128) on all host cores, one full solve per step (the reference's
    Fortran cannot be built here)."""
    rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import oracle
    from parcel_b import problems
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    if args.workload == "ddcg160":
        A, b, _ = problems.poisson3d_reference(160, 160, 160)
        kw = dict(solver=1, itrmax=2000, rtolmax=1e-9, ipreflag=2, ILU_method=1, precon_thblock=80)
        metric, workload = DD_METRIC, ("CG + block-Jacobi D-ILU (ILUD), 80 blocks, 160^3 Poisson (problem.f90), "
                                       "PRECISION_A/b/x/PRECONDITION = 2, rtol 1e-9")
    else:
        A, b = problem()
        kw = dict(solver=3, itrmax=3000, rtolmax=1e-10, ipreflag=2, ILU_method=1, precon_thblock=NBLOCKS,
                  GMRES_m=GMRES_M, GMRES_GSflag=1)
        metric, workload = DDG_METRIC, (f"dd GMRES({GMRES_M}) MGS + block-Jacobi D-ILU (ILUD), {NBLOCKS} blocks, "
                                        f"3D 7-pt upwind convection-diffusion {N_GRID}^3, b~N(0,1), "
                                        "PRECISION_A/b/x/PRECONDITION = 2, rtol 1e-10")
    times, niter, iret = [], 0, 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        _, _, _, niter, iret = oracle.ddcg(A, b, **kw)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    value = sum(times) / len(times)
    out = {"impl": "reference", "metric": metric, "value": value, "unit": "s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "double-double (pairs of f64)", "data": "synthetic",
           "config": {"workload": workload, "n": A.n, "nnz": A.nnz},
           "iterations": niter, "iret": iret,
           "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port",
                            "sample": "full solves of the same workload by the C++/OpenMP restatement of the "
                                      "reference's dd solver (its Fortran cannot be built here)"},
           "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_kernels_only(args):
    """Times the SpMV and the block-Jacobi ILU(0) application of the benchmark workload
    (CUDA events on the library stream), without solving; used for kernel profiles."""
    import torch
    from parcel_b import _lib, api
    L = _lib.load()
    A, b = problem()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    rp, ci, va = t(A.rowptr), t(A.col), t(A.val)
    ms_spmv, ms_pre = C.c_double(0), C.c_double(0)
    p = _lib.new_input(solver=3, ipreflag=1 if args.natural else 2, ILU_method=args.ilu_method,
                       precon_thblock=NBLOCKS, GMRES_m=GMRES_M)
    rc = L.parcel_b_bench_kernels(C.byref(p), C.byref(api.crs_struct(A, rp, ci, va)), args.steps,
                                  C.byref(ms_spmv), C.byref(ms_pre))
    assert rc == 0, _lib.last_error()
    diag = 0
    if args.natural:
        # point Jacobi keeps the natural layout, where the 7-point stencil's product runs on
        # its diagonal copy: 7 values + x + y per row (no column indices)
        spmv_bytes = 8 * 7 * A.n + 16 * A.n
        r = api.solve(A, t(b), rowptr=rp, col=ci, val=va, solver=3, ipreflag=1, GMRES_m=GMRES_M, itrmax=2,
                      rtolmax=RTOL)
        diag = r["stats"]["spmv_diagonals"]
    else:
        spmv_bytes = 12 * A.nnz + 4 * (A.n + 1) + 16 * A.n
    print(json.dumps({"spmv_us": ms_spmv.value * 1e3, "precon_us": ms_pre.value * 1e3,
                      "spmv_gbs": spmv_bytes / (ms_spmv.value * 1e-3) / 1e9, "spmv_bytes": spmv_bytes,
                      "layout": "natural, diagonal copy" if args.natural else "block-Jacobi level order, SELL",
                      "spmv_diagonals": diag,
                      "reps": args.steps}))


def run_network_only(args):
    """The learned stage's network alone (for kernel profiles): a handle for a 256^3 grid
    coarsened by 4 (64^3 coarse voxels), two forward passes on random inputs, CUDA-event
    time of the second."""
    import torch
    from parcel_b import _lib, api
    L = _lib.load()
    net = api.Learned(256, 256, 256, 4, seed=1)
    V = 64 ** 3
    u = torch.randn(V * 2, dtype=torch.float32, device="cuda")
    y = torch.zeros(V, dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(L.parcel_b_get_stream(), device=torch.device("cuda", 0))
    ms = []
    for _ in range(2):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        assert L.parcel_b_learned_forward(net.handle, 1, u.data_ptr(), y.data_ptr()) == 0, _lib.last_error()
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    flops = 2.0 * V * 27 * (2 * 32 + 4 * 32 * 32 + 32)
    print(json.dumps({"network_forward_ms": ms[-1], "coarse_voxels": V, "tflops": flops / (ms[-1] * 1e-3) / 1e12}))


def run_learned_only(args):
    """One learned-stage solve for kernel profiles: 256^3 variable-coefficient diffusion,
    FP32 FGMRES(40) inside FP64 refinement, BJ-ILU(0) 64 blocks, Galerkin coarse stage with
    --coarse-steps PCG steps from an untrained network's guess (the stage's cost does not
    depend on the weights), stopped after --itrmax inner iterations."""
    import torch
    from parcel_b import _lib, api, problems
    N, c = args.grid, args.coarsen
    g = problems.gaussian_random_field(N, corr_len=8.0, variance=2.0, seed=5)
    A = problems.vardiff3d(N, np.exp(g))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    rp, ci, va, bd = t(A.rowptr), t(A.col), t(A.val), t(problems.rhs_normal(A.n, 1000))
    net = api.Learned(N, N, N, c, seed=1)
    net.set_stage(args.coarse_steps, 1)
    L = _lib.load()
    p = _lib.new_input(solver=3, ipreflag=2, ILU_method=0, precon_thblock=NBLOCKS, GMRES_m=args.restart,
                       GMRES_GSflag=1, itrmax=args.itrmax, rtolmax=RTOL, inner_precision=1, inner_rtol=1e-4,
                       max_refine=80)
    S = api.crs_struct(A, rp, ci, va)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    niter, iret = C.c_int(0), C.c_int(0)
    t0 = time.perf_counter()
    rc = L.parcel_b_solve_learned(C.byref(p), C.byref(S), net.handle, bd.data_ptr(), x.data_ptr(), None,
                                  C.byref(niter), C.byref(iret))
    torch.cuda.synchronize()
    assert rc == 0, _lib.last_error()
    st = _lib.last_stats()
    print(json.dumps({"iterations": niter.value, "iret": iret.value, "wall_s": time.perf_counter() - t0,
                      "setup_s": st["setup_s"], "solve_s": st["solve_s"], "kernel_launches": st["kernel_launches"]}))


VD_METRIC = "time-to-1e-10 true rel. residual (s), learned + mixed-precision FGMRES vs plain FP64 PGMRES/BJ-ILU"


def vardiff_compare(N, c, m, nr, plain_rhs, train_rhs, train_steps, k=2, reps=5):
    """The learned-preconditioner workload: 3D 7-point variable-coefficient diffusion on an
    N^3 grid (N = 256 by default), coefficient exp(g) with g a Gaussian random field
    (correlation length 8 cells, variance 2, seed 5), harmonic-mean faces; right-hand
    sides N(0,1).  Arms, per right-hand side, every array already on the GPU, set-up
    included and amortised over the right-hand sides of one call:
      plain_fp64        FP64 PGMRES(m) + block-Jacobi ILU(0), 64 blocks (parcel_b_setup / _start)
      mixed_no_stage    FP32 FGMRES(m) + FP32 BJ-ILU(0) in FP64 refinement (parcel_b_solve_learned_many)
      mixed_coarse      the same + the Galerkin coarse stage, k coarse PCG steps from zero
      learned           the same + the coarse stage started from the trained network's guess
      mixed_coarse_k8   the coarse stage without the network at 8 coarse PCG steps
    The network is trained beforehand on pairs from plain solves with other right-hand
    sides (training time reported separately).  Time: CUDA events on the library stream
    around each synchronous call; the FGMRES arms report the median of `reps` calls (host
    hiccups such as a slow graph instantiation land in single calls), the plain arm one
    call."""
    import torch
    from parcel_b import _lib, api, problems
    L = _lib.load()
    g = problems.gaussian_random_field(N, corr_len=8.0, variance=2.0, seed=5)
    A = problems.vardiff3d(N, np.exp(g))
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rp, ci, va = t(A.rowptr), t(A.col), t(A.val)
    S = api.crs_struct(A, rp, ci, va)
    stream = torch.cuda.ExternalStream(L.parcel_b_get_stream(), device=dev)
    common = dict(solver=3, ipreflag=2, ILU_method=0, precon_thblock=NBLOCKS, GMRES_m=m, GMRES_GSflag=1,
                  itrmax=20000, rtolmax=RTOL)
    hist = np.zeros(20000)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, out

    # training on other right-hand sides
    t0 = time.perf_counter()
    net = api.Learned(N, N, N, c, seed=1)
    for sd in range(100, 100 + train_rhs):
        net.collect(A, problems.rhs_normal(A.n, sd), max_pairs=64, **common)
    t_collect = time.perf_counter() - t0
    t0 = time.perf_counter()
    f_loss, l_loss = net.train(steps=train_steps, batch=4, lr=2e-3, seed=3)
    t_train = time.perf_counter() - t0

    B = t(np.stack([problems.rhs_normal(A.n, 1000 + j) for j in range(nr)]))
    X = torch.zeros_like(B)
    it = np.zeros(nr, np.int32)
    ir = np.zeros(nr, np.int32)
    Asp = torch.sparse_csr_tensor((rp - 1).long(), (ci - 1).long(), va, size=(A.n, A.n))

    def plain_all(k_rhs):
        """plain FP64 PGMRES: one set-up (parcel_b_setup), then parcel_b_start per RHS"""
        p = _lib.new_input(**common)
        h = C.c_void_p()
        ts, its, rels = [], [], []
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s0.record(stream)
        assert L.parcel_b_setup(C.byref(p), C.byref(S), C.byref(h)) == 0, _lib.last_error()
        s1.record(stream)
        s1.synchronize()
        setup = s0.elapsed_time(s1) / 1e3
        for j in range(k_rhs):
            X[j].zero_()
            n_, i_ = C.c_int(0), C.c_int(0)
            dt, rc = timed(lambda: L.parcel_b_start(h, B[j].data_ptr(), X[j].data_ptr(), hist.ctypes.data,
                                                    C.byref(n_), C.byref(i_)))
            assert rc == 0, _lib.last_error()
            ts.append(dt)
            its.append(n_.value)
            rels.append(float(torch.linalg.norm(B[j] - Asp @ X[j]) / torch.linalg.norm(B[j])))
        L.parcel_b_release(h)
        return {"setup_s": setup, "solve_s_per_rhs": sum(ts) / len(ts), "rhs": len(ts), "iterations": its,
                "true_relres_max": max(rels), "fallbacks": 0,
                "s_per_rhs_amortised": setup / nr + sum(ts) / len(ts)}

    def fgmres_all(h, inner=1, n_rep=reps):
        """flexible GMRES (mixed precision when inner = 1), all RHS in one call, one set-up;
        the median of n_rep calls"""
        p = _lib.new_input(inner_precision=inner, inner_rtol=1e-4, max_refine=80, **common)
        calls = []
        for _ in range(n_rep):
            X.zero_()
            dt, rc = timed(lambda: L.parcel_b_solve_learned_many(C.byref(p), C.byref(S), h, nr, B.data_ptr(),
                                                                 X.data_ptr(), it.ctypes.data, ir.ctypes.data))
            assert rc == 0, _lib.last_error()
            calls.append((dt, _lib.last_stats()))
        rel = max(float(torch.linalg.norm(B[j] - Asp @ X[j]) / torch.linalg.norm(B[j])) for j in range(nr))
        dt, st = sorted(calls, key=lambda q: q[0])[len(calls) // 2]
        return {"setup_s": st["setup_s"], "solve_s_per_rhs": st["solve_s"] / nr, "rhs": nr,
                "iterations": it.tolist(), "true_relres_max": rel, "fallbacks": st["fallback"],
                "refine_steps": st["refine_steps"], "s_per_rhs_amortised": dt / nr, "call_s": dt,
                "calls_s": [round(q[0], 4) for q in calls]}

    # warm-up (graph capture, allocations) on a call of each FGMRES path
    fgmres_all(None, n_rep=1)
    net.set_stage(k, 1)
    fgmres_all(net.handle, n_rep=1)
    clk = Clocks(0)
    clk.started()
    sp = plain_all(min(plain_rhs, nr))
    sm = fgmres_all(None)
    net.set_stage(k, 0)
    sc = fgmres_all(net.handle)
    net.set_stage(k, 1)
    sl = fgmres_all(net.handle)
    net.set_stage(8, 0)
    s8 = fgmres_all(net.handle)
    clocks = clk.stop()
    mean = lambda r: float(np.mean(r["iterations"]))
    out = {"metric": VD_METRIC, "value": sl["call_s"], "unit": "s", "n_gpus": 1,
           "steps": nr, "warmup": 1, "ms_per_step": sl["s_per_rhs_amortised"] * 1e3, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 refinement, bf16 network",
           "data": "synthetic",
           "config": {"workload": f"variable-coefficient 7-pt diffusion {N}^3, k=exp(GRF(corr 8, var 2)), "
                                  f"{nr} RHS N(0,1), FGMRES({m}) + BJ-ILU(0) {NBLOCKS} blocks + Galerkin coarse "
                                  f"stage on the {N // c}^3 grid ({k} coarse PCG steps, network guess), "
                                  f"tol {RTOL}",
                      "n": A.n, "nnz": A.nnz, "coarsen": c, "coarse_steps": k, "l2": "inputs larger than L2"},
           "plain_fp64": sp, "mixed_no_stage": sm, "mixed_coarse": sc, "learned": sl, "mixed_coarse_k8": s8,
           "speedup_vs_plain_fp64": sp["s_per_rhs_amortised"] / sl["s_per_rhs_amortised"],
           "speedup_mixed_vs_plain_fp64": sp["s_per_rhs_amortised"] / sm["s_per_rhs_amortised"],
           "network_gain": {"iterations_without": mean(sc), "iterations_with": mean(sl),
                            "time_ratio": sc["s_per_rhs_amortised"] / sl["s_per_rhs_amortised"],
                            "vs_coarse_k8_time_ratio": s8["s_per_rhs_amortised"] / sl["s_per_rhs_amortised"]},
           "training": {"pairs": net.num_pairs(), "collect_s": t_collect, "train_s": t_train,
                        "steps": train_steps, "loss_first": f_loss, "loss_last": l_loss},
           "clocks": clocks}
    return out


def run_vardiff(args):
    print(json.dumps(vardiff_compare(args.grid, args.coarsen, args.restart, args.rhs, args.plain_rhs,
                                     args.train_rhs, args.train_steps, k=args.coarse_steps)))


DD_METRIC = "time to 1e-9 recursive rel. residual (s), double-double PCG + block-Jacobi D-ILU"


def run_ddcg(args):
    """The reference's double-double CG configuration (template_cpu/STDOUT_run_dd): 160^3
    Poisson of src/example/problem.f90, CG with block-Jacobi D-ILU (ILUD), 80 blocks, every
    PRECISION_* = 2, rtol 1e-9, x0 = 0.  value: the whole parcel_b_ddcg call with the
    arrays in HBM (CUDA events on the library stream); e2e: parcel_ddcg_c_ with host arrays
    (copies in and out inside the timed region); cpu_baseline: the oracle's C++/OpenMP
    restatement of ddKSP_pCG, one full solve.  The reference's own CPU run printed a CRS
    solve time of 3.79 s with 4 MPI ranks x 20 OpenMP threads on its authors' machine."""
    import torch
    from parcel_b import _lib, api, problems
    L = _lib.load()
    A, b, xe = problems.poisson3d_reference(160, 160, 160)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rp, ci, va, bd = t(A.rowptr), t(A.col), t(A.val), t(b)
    stream = torch.cuda.ExternalStream(L.parcel_b_get_stream(), device=dev)
    kw = dict(itrmax=2000, rtolmax=1e-9, ipreflag=2, ILU_method=1, precon_thblock=80)

    def solve_dev():
        return api.ddcg(A, bd, rowptr=rp, col=ci, val=va, **kw)

    for _ in range(args.warmup):
        res = solve_dev()
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.started()
    times = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = solve_dev()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    clocks = clk.stop()
    x = res["x_hi"].cpu().numpy() + res["x_lo"].cpu().numpy()
    err = float(np.abs(x - xe).max())
    # end to end through the reference-ordered C shim with pinned host arrays
    hp = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_rp, h_ci, h_va, h_b = hp(A.rowptr), hp(A.col), hp(A.val), hp(b)
    zeros = lambda m: torch.zeros(m, dtype=torch.float64).pin_memory().numpy()
    h_x, h_xl, h_bl, h_al = zeros(A.n), zeros(A.n), zeros(A.n), zeros(A.nnz)
    hist = np.zeros(2000)
    I = lambda v: C.byref(C.c_int(v))
    i32 = lambda v: C.byref(C.c_int32(v))
    ptr = lambda a: a.ctypes.data

    def solve_host():
        h_x[:] = 0.0
        h_xl[:] = 0.0
        niter, iret = C.c_int(2000), C.c_int(0)
        L.parcel_ddcg_c_(I(0), ptr(h_x), ptr(h_xl), ptr(h_b), ptr(h_bl), i32(A.n), i32(A.n), i32(A.nnz), i32(1),
                         ptr(h_va), ptr(h_al), ptr(h_rp), ptr(h_ci), I(2), I(1), I(0), I(1), C.byref(niter),
                         C.byref(C.c_double(1e-9)), ptr(hist), I(0), I(80), I(1), I(1), I(2000), I(2), I(2), I(2),
                         I(2), C.byref(iret))
        return niter.value, iret.value

    solve_host()
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        solve_host()
        e2e.append(time.perf_counter() - t0)
    out = {"metric": DD_METRIC, "value": sum(times) / len(times), "unit": "s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "double-double (pairs of f64)", "data": "synthetic",
           "config": {"workload": "CG + block-Jacobi D-ILU (ILUD), 80 blocks, 160^3 Poisson (problem.f90), "
                                  "PRECISION_A/b/x/PRECONDITION = 2, rtol 1e-9",
                      "n": A.n, "nnz": A.nnz, "l2": "inputs larger than L2 (dd vectors 65 MB each + matrix)"},
           "iterations": res["niter"], "iret": res["iret"], "max_abs_err": err,
           "step_times_s": [round(v, 6) for v in times],
           "e2e": {"value": sum(e2e) / len(e2e), "unit": "s",
                   "h2d_bytes_per_step": int(A.rowptr.nbytes + A.col.nbytes + 2 * A.val.nbytes + 4 * A.n * 8),
                   "d2h_bytes_per_step": int(2 * A.n * 8 + res["niter"] * 8)},
           "reference_printed_solve_s": 3.79280038102297, "clocks": clocks}
    if not args.no_cpu_baseline:
        import oracle
        t0 = time.perf_counter()
        _, _, h, niter, iret = oracle.ddcg(A, b, **kw)
        out["cpu_baseline"] = {"value": time.perf_counter() - t0, "unit": "s", "cores": oracle.num_threads(),
                               "kind": "port", "sample": f"one full oracle solve ({niter} iterations, iret {iret})"}
    print(json.dumps(out))


DDG_METRIC = "time to 1e-10 rel. residual (s), double-double GMRES(30) + block-Jacobi D-ILU"


def run_ddgmres(args):
    """Double-double GMRES(30), MGS, block-Jacobi D-ILU (ILUD) with 64 blocks, every
    PRECISION_* = 2, on the FP64 line's matrix (3D 7-point upwind convection-diffusion
    128^3, b ~ N(0,1)), rtol 1e-10.  value: the whole parcel_b_ddgmres call with the arrays
    in HBM (CUDA events on the library stream); e2e: parcel_ddgmres_c_ with pinned host
    arrays; cpu_baseline: the oracle's restatement of ddKSP_pGMRES on two restart cycles
    (60 iterations), scaled to the GPU's iteration count.  The reference publishes no time
    for its dd GMRES."""
    import torch
    from parcel_b import _lib, api
    L = _lib.load()
    A, b = problem()
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rp, ci, va, bd = t(A.rowptr), t(A.col), t(A.val), t(b)
    stream = torch.cuda.ExternalStream(L.parcel_b_get_stream(), device=dev)
    itrmax = 3000
    kw = dict(itrmax=itrmax, rtolmax=1e-10, ipreflag=2, ILU_method=1, precon_thblock=NBLOCKS, GMRES_m=GMRES_M,
              GMRES_GSflag=1)

    def solve_dev():
        return api.ddgmres(A, bd, rowptr=rp, col=ci, val=va, **kw)

    for _ in range(args.warmup):
        res = solve_dev()
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.started()
    times = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = solve_dev()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    clocks = clk.stop()
    import oracle
    x = res["x_hi"].cpu().numpy() + res["x_lo"].cpu().numpy()
    relres = oracle.true_relres(A, b, x)
    hp = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_rp, h_ci, h_va, h_b = hp(A.rowptr), hp(A.col), hp(A.val), hp(b)
    zeros = lambda m: torch.zeros(m, dtype=torch.float64).pin_memory().numpy()
    h_x, h_xl, h_bl, h_al = zeros(A.n), zeros(A.n), zeros(A.n), zeros(A.nnz)
    hist = np.zeros(itrmax)
    I = lambda v: C.byref(C.c_int(v))
    i32 = lambda v: C.byref(C.c_int32(v))
    ptr = lambda a: a.ctypes.data

    def solve_host():
        h_x[:] = 0.0
        h_xl[:] = 0.0
        niter, iret = C.c_int(itrmax), C.c_int(0)
        L.parcel_ddgmres_c_(I(0), ptr(h_x), ptr(h_xl), ptr(h_b), ptr(h_bl), i32(A.n), i32(A.n), i32(A.nnz), i32(1),
                            ptr(h_va), ptr(h_al), ptr(h_rp), ptr(h_ci), I(2), I(1), I(0), I(1), C.byref(niter),
                            C.byref(C.c_double(1e-10)), ptr(hist), I(0), I(NBLOCKS), I(1), I(1), I(2000),
                            I(GMRES_M), I(1), I(2), I(2), I(2), I(2), C.byref(iret))
        return niter.value, iret.value

    solve_host()
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        solve_host()
        e2e.append(time.perf_counter() - t0)
    out = {"metric": DDG_METRIC, "value": sum(times) / len(times), "unit": "s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "double-double (pairs of f64)", "data": "synthetic",
           "config": {"workload": f"dd GMRES({GMRES_M}) MGS + block-Jacobi D-ILU (ILUD), {NBLOCKS} blocks, "
                                  f"3D 7-pt upwind convection-diffusion {N_GRID}^3, b~N(0,1), "
                                  "PRECISION_A/b/x/PRECONDITION = 2, rtol 1e-10",
                      "n": A.n, "nnz": A.nnz, "l2": "inputs larger than L2 (dd vectors 34 MB each, basis 1 GB)"},
           "iterations": res["niter"], "iret": res["iret"], "true_relres": relres,
           "step_times_s": [round(v, 6) for v in times],
           "e2e": {"value": sum(e2e) / len(e2e), "unit": "s",
                   "h2d_bytes_per_step": int(A.rowptr.nbytes + A.col.nbytes + 2 * A.val.nbytes + 4 * A.n * 8),
                   "d2h_bytes_per_step": int(2 * A.n * 8 + res["niter"] * 8)},
           "clocks": clocks}
    if not args.no_cpu_baseline:
        sample = 2 * GMRES_M
        t0 = time.perf_counter()
        _, _, h, niter, iret = oracle.ddcg(A, b, solver=3, **dict(kw, itrmax=sample))
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": el * res["niter"] / max(niter, 1), "unit": "s", "cores": oracle.num_threads(),
                               "kind": "port",
                               "sample": f"the oracle's dd GMRES on the same workload for {niter} iterations "
                                         f"({el:.1f} s, set-up included), scaled to {res['niter']} iterations"}
    print(json.dumps(out))



# ---------------------------------------------------------------- configurations C1, C3, C4
CFG_METRIC = "time to the configuration's tolerance (s): true rel. residual for GMRES-type solves, recursive for CG"


def _cfg(name):
    """The three further configurations of the hot path, each with its solver options, the
    reference-facing entry used for the end-to-end time, the kernels that bound it and the
    oracle solve that times the reference's algorithm on the host."""
    from parcel_b import problems
    if name == "poisson2d256":
        A = problems.poisson2d_5pt(256, 256)
        b = problems.rhs_uniform(A.n, 1)
        return dict(A=A, b=b, shim="parcel_dcg", dtype="f64",
                    workload="PCG FP64 + point Jacobi, 2D 5-pt Poisson 256^2 (4 / -1, Dirichlet), b~U[-1,1), "
                             "x0=0, rtol 1e-8 (recursive residual)",
                    opts=dict(solver=1, ipreflag=1, itrmax=5000, rtolmax=1e-8),
                    shim_args=dict(ipreflag=1, ILU_method=0), kern=dict(ipreflag=1), dominant="spmv",
                    l2="5.2 MB per SpMV: L2-resident, launch-bound (not scored against HBM)")
    if name == "aniso192":
        A = problems.aniso3d(192, k=(1.0, 1e-2, 1e-4))
        b = problems.rhs_uniform(A.n, 3)
        opts = dict(solver=1, ipreflag=2, ILU_method=0, precon_thblock=64, itrmax=20000, rtolmax=1e-12,
                    inner_precision=1, residual_dd=1, inner_rtol=1e-4, max_refine=80)
        return dict(A=A, b=b, shim=None, dtype="f32 inner / f64 + dd refinement",
                    workload="mixed precision: FP32 PCG + FP32 block-Jacobi ILU(0) 64 blocks inside FP64 / "
                             "double-double refinement, anisotropic 7-pt (1, 1e-2, 1e-4) 192^3, b~U[-1,1), "
                             "stop at FP64 true rel. residual 1e-12",
                    opts=opts, kern=dict(ipreflag=2, ILU_method=0, precon_thblock=64, inner_precision=1),
                    dominant="precon", l2="inputs larger than L2 (FP32 matrix 394 MB)")
    if name == "banded4m":
        A = problems.banded_random(4_000_000, bandwidth=64, nnz_row=9, seed=4)
        b = problems.rhs_normal(A.n, 4)
        return dict(A=A, b=b, shim="parcel_dcagmres", dtype="f64",
                    workload="CA-GMRES(s=8, t=8: restart 64) FP64, Newton basis with Leja-ordered Ritz shifts, "
                             "TSQR, point Jacobi, random banded nonsymmetric n=4,000,000 (9 nnz/row in |i-j|<=64, "
                             "diagonal 1.2 x row abs sum), b~N(0,1), tol 1e-10",
                    opts=dict(solver=4, CAGMRES_sstep=8, CAGMRES_tstep=8, CAGMRES_basis=1, CAGMRES_QRflag=3,
                              ipreflag=1, itrmax=3000, rtolmax=1e-10),
                    shim_args=dict(ipreflag=1, ILU_method=0, CAGMRES_sstep=8, CAGMRES_tstep=8, CAGMRES_basis=1,
                                   CAGMRES_QRflag=3),
                    kern=dict(ipreflag=1), dominant="spmv", l2="inputs larger than L2 (512 MB per SpMV)")
    raise ValueError(name)


def _cfg_oracle(name, c, max_s=None):
    """The reference's algorithm on the host: the C++/OpenMP oracle (PCG, block-Jacobi ILU,
    point Jacobi) or the numpy CA-GMRES restatement.  Returns (seconds, niter, iret, x,
    cores, sample)."""
    import oracle
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    A, b = c["A"], c["b"]
    if name == "banded4m":
        import cagmres
        t0 = time.perf_counter()
        x, h, niter, iret = cagmres.pcagmres(A, b, s=8, t=8, basis=1, qrflag=3, itrmax=3000, rtolmax=1e-10,
                                             ipreflag=1)
        return (time.perf_counter() - t0, niter, iret, x, 1,
                "one full solve by the numpy restatement of KSP_pCAGMRES (scipy SpMV, one core)")
    kw = dict(c["opts"])
    for k in ("inner_precision", "residual_dd", "inner_rtol", "max_refine"):
        kw.pop(k, None)
    reps = 20 if name == "poisson2d256" else 1
    M = oracle.Matrix(A)
    t0 = time.perf_counter()
    for _ in range(reps):
        x, h, niter, iret = oracle.solve(M, b, **kw)
    dt = (time.perf_counter() - t0) / reps
    what = "FP64 PCG + block-Jacobi ILU(0) to 1e-12" if name == "aniso192" else "PCG + point Jacobi"
    return (dt, niter, iret, x, cores,
            f"{reps} full solve(s) by the C++/OpenMP restatement ({what}), mean time per solve")


def run_config(args):
    import torch
    from parcel_b import _lib, api
    name = args.workload
    L = _lib.load()
    c = _cfg(name)
    A, b = c["A"], c["b"]
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rp, ci, va, bd = t(A.rowptr), t(A.col), t(A.val), t(b)
    stream = torch.cuda.ExternalStream(L.parcel_b_get_stream(), device=dev)
    itrmax = c["opts"]["itrmax"]
    hist = np.zeros(itrmax)
    x = torch.zeros(A.n, dtype=torch.float64, device=dev)
    S_dev = api.crs_struct(A, rp, ci, va)

    def solve_dev():
        x.zero_()
        if c["shim"]:
            fn = getattr(api, c["shim"])
            n_, i_ = fn(x, bd, A.n, A.n, A.nnz, 1, va, rp, ci, addL=0, iflagAS=1, itrmax=itrmax,
                        rtolmax=c["opts"]["rtolmax"], reshistory=hist, **c["shim_args"])
            return n_, i_, _lib.last_stats()
        p_ = _lib.new_input(**c["opts"])
        n_, i_ = C.c_int(0), C.c_int(0)
        rc_ = L.parcel_b_solve(C.byref(p_), C.byref(S_dev), bd.data_ptr(), x.data_ptr(), hist.ctypes.data,
                               C.byref(n_), C.byref(i_))
        assert rc_ == 0, _lib.last_error()
        return n_.value, i_.value, _lib.last_stats()

    for _ in range(args.warmup):
        solve_dev()
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.started()
    times, stats = [], None
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        niter, iret, stats = solve_dev()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    clocks = clk.stop()
    xg = x.cpu().numpy()
    import oracle
    relres = oracle.true_relres(A, b, xg)

    # end to end: pinned host arrays through the reference-facing entry (the C shim, or
    # parcel_b_solve for the mixed-precision extension), copies inside the timed region
    hp = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_rp, h_ci, h_va, h_b = hp(A.rowptr), hp(A.col), hp(A.val), hp(b)
    h_x = torch.zeros(A.n, dtype=torch.float64).pin_memory().numpy()

    def solve_host():
        h_x[:] = 0.0
        if c["shim"]:
            fn = getattr(api, c["shim"])
            return fn(h_x, h_b, A.n, A.n, A.nnz, 1, h_va, h_rp, h_ci, addL=0, iflagAS=1, itrmax=itrmax,
                      rtolmax=c["opts"]["rtolmax"], reshistory=hist, **c["shim_args"])
        Ah = type(A)(n=A.n, rowptr=h_rp, col=h_ci, val=h_va)
        p_ = _lib.new_input(**c["opts"])
        n_, i_ = C.c_int(0), C.c_int(0)
        rc_ = L.parcel_b_solve(C.byref(p_), C.byref(api.crs_struct(Ah)), h_b.ctypes.data, h_x.ctypes.data,
                               hist.ctypes.data, C.byref(n_), C.byref(i_))
        assert rc_ == 0, _lib.last_error()
        return n_.value, i_.value

    solve_host()
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        solve_host()
        e2e.append(time.perf_counter() - t0)

    # the kernels that bound the iteration (CUDA events on the library stream)
    ms_spmv, ms_pre = C.c_double(0), C.c_double(0)
    p = _lib.new_input(**c["kern"])
    rc = L.parcel_b_bench_kernels(C.byref(p), C.byref(api.crs_struct(A, rp, ci, va)), 50, C.byref(ms_spmv),
                                  C.byref(ms_pre))
    assert rc == 0, _lib.last_error()
    hbm, peak_kind = peaks()
    f32 = c["kern"].get("inner_precision", 0) == 1
    vb = 4 if f32 else 8
    spmv_bytes = (vb + 4) * A.nnz + 4 * (A.n + 1) + 2 * vb * A.n
    # block-Jacobi ILU: L and U values and columns, row pointers, r read, z written twice
    pre_bytes = (vb + 4) * A.nnz + 8 * (A.n + 1) + 4 * vb * A.n if c["dominant"] == "precon" else 3 * 8 * A.n
    if c["dominant"] == "spmv":
        rk, rb, rt = ("k_spmv_sell<double,double> (sliced-ELLPACK SpMV)", spmv_bytes, ms_spmv.value)
    else:
        rk, rb, rt = ("k_ilu_sweep_grp<float> (block-Jacobi ILU(0) forward + backward sweep, FP32)", pre_bytes,
                      ms_pre.value)
    ach = rb / (rt * 1e-3) / 1e9
    value = sum(times) / len(times)
    out = {"metric": CFG_METRIC, "value": value, "unit": "s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": c["dtype"], "data": "synthetic",
           "config": {"workload": c["workload"], "n": A.n, "nnz": A.nnz, "l2": c["l2"]},
           "iterations": niter, "iret": iret, "true_relres": relres,
           "step_times_s": [round(v, 6) for v in times],
           "setup_s": stats["setup_s"], "solve_s": stats["solve_s"],
           "e2e": {"value": sum(e2e) / len(e2e), "unit": "s",
                   "h2d_bytes_per_step": int(A.rowptr.nbytes + A.col.nbytes + A.val.nbytes + 2 * A.n * 8),
                   "d2h_bytes_per_step": int(A.n * 8 + itrmax * 8)},
           "roofline": {"bound": "hbm", "kernel": rk, "achieved": ach, "peak": hbm, "unit": "GB/s",
                        "frac": ach / hbm, "peak_kind": peak_kind, "traffic": None, "algorithmic_bytes": int(rb),
                        "us_per_launch": rt * 1e3},
           "kernels_us": {"spmv": ms_spmv.value * 1e3, "precon_apply": ms_pre.value * 1e3},
           "clocks": clocks, "gpu_launches": int(stats["kernel_launches"])}
    if name == "aniso192":
        out["refine_steps"] = stats["refine_steps"]
        out["true_relres_dd"] = stats["true_relres_dd"]
        # the plain FP64 GPU path on the same system, for the mixed-precision gain
        kw = {k: v for k, v in c["opts"].items() if k not in ("inner_precision", "residual_dd", "inner_rtol",
                                                                "max_refine")}
        api.solve(A, bd, rowptr=rp, col=ci, val=va, **kw)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r64 = api.solve(A, bd, rowptr=rp, col=ci, val=va, **kw)
        e1.record(stream)
        e1.synchronize()
        out["plain_fp64_gpu"] = {"s": e0.elapsed_time(e1) / 1e3, "iterations": r64["niter"],
                                 "true_relres": oracle.true_relres(A, b, r64["x"].cpu().numpy())}
        # double-double reference solution: the library's dd CG with D-ILU (bit-identical to the
        # oracle's dd CG in the tests), run to a dd recursive residual of 1e-24
        rdd = api.ddcg(A, bd, rowptr=rp, col=ci, val=va, itrmax=20000, rtolmax=1e-24, ipreflag=2, ILU_method=1,
                       precon_thblock=64)
        xdd_hi, xdd_lo = rdd["x_hi"].cpu().numpy(), rdd["x_lo"].cpu().numpy()
        scale = np.abs(xdd_hi).max()
        out["error_vs_dd_reference"] = {
            "max_abs_rel": float(np.abs((xg - xdd_hi) - xdd_lo).max() / scale),
            "dd_solve": f"dd CG + D-ILU 64 blocks, {rdd['niter']} iterations, dd recursive residual 1e-24"}
    if not args.no_cpu_baseline:
        dt, no, io, xo, cores, sample = _cfg_oracle(name, c)
        out["cpu_baseline"] = {"value": dt, "unit": "s", "cores": cores,
                               "kind": "port", "sample": sample + f" ({no} iterations, iret {io})"}
        out["oracle_iterations"] = no
        if name == "aniso192":
            out["error_vs_fp64_oracle"] = {"max_abs_rel": float(np.abs(xg - xo).max() / np.abs(xo).max()),
                                           "oracle_true_relres": oracle.true_relres(A, b, xo)}
    print(json.dumps(out))


def run_reference_config(args):
    rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        return
    name = args.workload
    c = _cfg(name)
    times, niter, iret, cores, sample = [], 0, 0, 1, ""
    for i in range(args.warmup + args.steps):
        dt, niter, iret, _, cores, sample = _cfg_oracle(name, c)
        if i >= args.warmup:
            times.append(dt)
    value = sum(times) / len(times)
    out = {"impl": "reference", "metric": CFG_METRIC, "value": value, "unit": "s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": c["workload"], "n": c["A"].n, "nnz": c["A"].nnz, "l2": c["l2"]},
           "iterations": niter, "iret": iret,
           "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


DDM_METRIC = "DDM CG solve time (s), 160^3 Poisson, block-Jacobi D-ILU on 4^3 boxes, rtol 1e-9"


def _ddm_problem():
    import ddm as oddm
    return oddm.poisson3d_ddm((160, 160, 160), (1, 1, 1), 0)


def run_ddm(args):
    """The reference's DDM example as its CUDA build runs it (src/example/main_ddm.f90,
    make_poisson_3D_DDM 160^3, CG, block-Jacobi D-ILU on 4^3 boxes (DDM_CUDA_BJ), rtol 1e-9,
    x0 = 0; template_gpu/STDOUT_run_ddm: 345 iterations and a printed solve time of 0.617 s
    with 4 processes of a y-split, whose boxes are the same 4^3 boxes).  One process holds
    the whole grid here.  value: the whole parcel_b_solve_ddm call (renumbering, set-up and
    solve, as the reference's timer brackets parcel_dcg_ddm) with the arrays in HBM, CUDA
    events on the library stream; e2e: the same call with pinned host arrays (copies inside
    the timed region); cpu_baseline: the oracle on the renumbered matrix (oracle/ddm.py), one
    full solve on all host cores; rooflines: the SpMV and the D-ILU sweep of the renumbered
    system (parcel_b_bench_kernels_ddm), with the byte models of the default line."""
    import torch
    from parcel_b import _lib, ddm
    L = _lib.load()
    p = _ddm_problem()
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    val, off, bd = t(p["val"]), t(p["offset"]), t(p["b"])
    stream = torch.cuda.ExternalStream(L.parcel_b_get_stream(), device=dev)
    kw = dict(boxes=ddm.BOXES_CUBES, solver=1, ipreflag=2, itrmax=2000, rtolmax=1e-9)

    def solve_dev():
        return ddm.solve(val, off, p["offset_dim"], p["n"], bd, **kw)

    for _ in range(args.warmup):
        res = solve_dev()
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.started()
    times = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = solve_dev()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    clocks = clk.stop()
    x = res["x"].cpu().numpy()
    err = float(np.abs(x - p["x_exact"]).max() / np.abs(p["x_exact"]).max())
    hist_dev = res["reshistory"]
    try:
        with open(os.path.join(ROOT, "tests", "golden", "reference_templates.json")) as f:
            g = np.array(json.load(f)["gpu_ddm_cg_cubes"]["history"])
        k = min(len(g), len(hist_dev))
        parity = {"template_iterations": len(g), "max_rel_history_diff": float(np.max(np.abs(hist_dev[:k] - g[:k]) / g[:k]))}
    except (OSError, KeyError):
        parity = None
    # end to end: the same call with pinned host arrays (x too: zero initial guess in, the
    # solution out, in place)
    hp = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_val, h_off, h_b, h_x = hp(p["val"]), hp(p["offset"]), hp(p["b"]), hp(np.zeros_like(p["b"]))
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        h_x[:] = 0.0
        t0 = time.perf_counter()
        ddm.solve(h_val, h_off, p["offset_dim"], p["n"], h_b, out=h_x, **kw)
        e2e.append(time.perf_counter() - t0)
    e2e_err = float(np.abs(h_x - p["x_exact"]).max() / np.abs(p["x_exact"]).max())
    # kernel rooflines on the renumbered system
    prm = _lib.new_input(solver=1, ipreflag=2)
    D = ddm.ddm_struct(val, off, p["offset_dim"], p["n"], boxes=ddm.BOXES_CUBES)
    ms_spmv, ms_pre = C.c_double(0), C.c_double(0)
    rc = L.parcel_b_bench_kernels_ddm(C.byref(prm), C.byref(D), 50, C.byref(ms_spmv), C.byref(ms_pre))
    if rc != 0:
        raise RuntimeError(f"parcel_b_bench_kernels_ddm failed: {_lib.last_error()}")
    n = int(np.prod(p["n"]))
    nnz = int(np.count_nonzero(p["val"]))
    hbm, peak_kind = peaks()
    spmv_bytes = 12 * nnz + 4 * (n + 1) + 16 * n
    ilu_bytes = 12 * nnz + 8 * (n + 1) + 32 * n
    sp_ach = spmv_bytes / (ms_spmv.value * 1e-3) / 1e9
    il_ach = ilu_bytes / (ms_pre.value * 1e-3) / 1e9
    m = p["m"]
    out = {"metric": DDM_METRIC, "value": sum(times) / len(times), "unit": "s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "DDM 160^3 Poisson (make_poisson_3D_DDM), CG + block-Jacobi D-ILU on 4^3 boxes, "
                                  "rtol 1e-9, one process", "n": n, "padded_cells": m, "nnz": nnz,
                      "l2": "inputs larger than L2 (the 7 x 4.4M-cell DIA values are 245 MB)"},
           "iterations": res["niter"], "iret": res["iret"], "max_rel_error": err, "parity": parity,
           "setup_s": res["stats"]["setup_s"], "solve_s": res["stats"]["solve_s"],
           "step_times_s": [round(v, 6) for v in times],
           "e2e": {"value": sum(e2e) / len(e2e), "unit": "s", "h2d_bytes_per_step": int(h_val.nbytes + h_off.nbytes + 2 * m * 8),
                   "d2h_bytes_per_step": int(m * 8 + res["niter"] * 8), "max_rel_error": e2e_err},
           "roofline": {"bound": "hbm", "kernel": "k_spmv_sell<double,double> on the renumbered system",
                        "achieved": sp_ach, "peak": hbm, "unit": "GB/s", "frac": sp_ach / hbm, "peak_kind": peak_kind,
                        "traffic": None, "algorithmic_bytes": int(spmv_bytes), "us_per_launch": ms_spmv.value * 1e3},
           "roofline_dominant": {"bound": "hbm", "kernel": "block-Jacobi D-ILU sweep over the 64,000 boxes",
                                 "achieved": il_ach, "peak": hbm, "unit": "GB/s", "frac": il_ach / hbm,
                                 "peak_kind": peak_kind, "algorithmic_bytes": int(ilu_bytes),
                                 "us_per_launch": ms_pre.value * 1e3},
           "reference_printed_solve_s": {"cuda_build_4_processes": 0.617148808203638,
                                         "cpu_build_4x20_threads_x_slabs": 1.58943619503407},
           "clocks": clocks, "gpu_launches": int(res["stats"]["kernel_launches"]) * args.steps}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = _ddm_oracle_run()
    print(json.dumps(out))


def _ddm_oracle_run():
    """The oracle's CG on the renumbered DDM system (all host threads): one full solve."""
    import ddm as oddm
    import oracle
    from parcel_b.problems import CRS
    p = _ddm_problem()
    G = oddm.global_system([p], (1, 1, 1), oddm.cube_boxes)
    A = CRS(n=G["n"], rowptr=G["rowptr"], col=G["col"], val=G["val"])
    t0 = time.perf_counter()
    _, h, niter, iret = oracle.solve(A, G["b"], solver=1, ipreflag=2, ILU_method=1, itrmax=2000, rtolmax=1e-9,
                                     blocks=G["starts"])
    return {"value": time.perf_counter() - t0, "unit": "s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"one full oracle solve of the renumbered system ({niter} iterations, iret {iret})"}


def run_reference_ddm(args):
    """Reference arm of the DDM line: the oracle's CPU restatement, one full solve per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    vals = [_ddm_oracle_run() for _ in range(max(1, args.steps))]
    v = sum(c["value"] for c in vals) / len(vals)
    out = {"impl": "reference", "metric": DDM_METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": 0, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "DDM 160^3 Poisson (make_poisson_3D_DDM), CG + block-Jacobi D-ILU on 4^3 boxes, "
                                  "rtol 1e-9, one process"},
           "cpu_baseline": dict(vals[-1], value=v),
           "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="default line without the GPU summary of the other configurations")
    ap.add_argument("--kernels-only", action="store_true")
    ap.add_argument("--network", action="store_true", help="with --kernels-only: the learned stage's network alone")
    ap.add_argument("--learned", action="store_true",
                    help="with --kernels-only: one learned-stage solve of --itrmax inner iterations")
    ap.add_argument("--itrmax", type=int, default=80)
    ap.add_argument("--natural", action="store_true",
                    help="with --kernels-only: point Jacobi, natural layout (the SpMV's diagonal copy)")
    ap.add_argument("--ilu-method", type=int, default=0)
    ap.add_argument("--workload", default="convdiff128",
                    choices=["convdiff128", "vardiff", "ddcg160", "ddgmres128", "poisson2d256", "aniso192",
                             "banded4m", "ddm160"],
                    help="vardiff: the learned-preconditioner comparison; ddcg160: the double-double CG "
                         "configuration of the reference's dd example; ddgmres128: the double-double GMRES "
                         "on the default line's matrix (none of them is the default line)")
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--coarsen", type=int, default=8)
    ap.add_argument("--restart", type=int, default=40)
    ap.add_argument("--rhs", type=int, default=16)
    ap.add_argument("--plain-rhs", type=int, default=16)
    ap.add_argument("--train-rhs", type=int, default=4)
    ap.add_argument("--coarse-steps", type=int, default=2,
                    help="coarse PCG steps of the learned stage (the mixed_coarse arm uses the same)")
    ap.add_argument("--train-steps", type=int, default=400)
    ap.add_argument("--target-rhs", type=int, default=2,
                    help="right-hand sides of the learned-preconditioner target on the default line (0: skip)")
    ap.add_argument("--target-train-rhs", type=int, default=2)
    ap.add_argument("--target-train-steps", type=int, default=400)
    args = ap.parse_args()
    if args.workload == "ddm160":
        run_reference_ddm(args) if args.impl == "reference" else run_ddm(args)
    elif args.impl == "reference" and args.workload in ("ddcg160", "ddgmres128"):
        run_reference_dd(args)
    elif args.impl == "reference" and args.workload == "vardiff":
        print(json.dumps({"impl": "reference", "unavailable": "the learned preconditioner has no counterpart in "
                                                              "the reference; its plain-preconditioner arm is part "
                                                              "of the vardiff line"}))
    elif args.workload in ("poisson2d256", "aniso192", "banded4m"):
        if args.impl == "reference":
            run_reference_config(args)
        else:
            run_config(args)
    elif args.workload == "vardiff":
        run_vardiff(args)
    elif args.workload == "ddcg160":
        run_ddcg(args)
    elif args.workload == "ddgmres128":
        run_ddgmres(args)
    elif args.kernels_only and args.network:
        run_network_only(args)
    elif args.kernels_only and args.learned:
        run_learned_only(args)
    elif args.kernels_only:
        run_kernels_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
