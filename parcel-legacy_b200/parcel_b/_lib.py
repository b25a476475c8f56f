"""Loader of libparcelb.so (the CUDA library) and ctypes declarations of include/parcel_b.h.

The library is built in-tree by parcel-legacy_b200/build.py.  There is no CPU fallback:
if the shared object is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "libparcelb.so")

# ---- constants mirrored from include/parcel_b.h (src/define.f90:14-102) ----
OK = 0
MAXITER = 1
E_ZERO_PIVOT = -1
E_ARG = -2
E_CUDA = -3
E_BREAKDOWN = -4
E_UNSUPPORTED = -5
E_NOMEM = -6
SOLVER_CG, SOLVER_BICG, SOLVER_GMRES, SOLVER_CAGMRES = 1, 2, 3, 4
PRECON_NONE, PRECON_PJ, PRECON_BJ, PRECON_AS = 0, 1, 2, 3
ILU0, ILUD, MLUD = 0, 1, 2
GS_MGS, GS_CGS = 1, 2
INNER_FP64, INNER_FP32_REFINE = 0, 1


class Input(C.Structure):
    """parcel_b_input == KSP_INPUT_PARAM (src/type.f90:907-946) + extensions."""
    _fields_ = [(n, C.c_int) for n in (
        "ipreflag", "ILU_method", "addL", "iflagAS", "solver", "iovlflag", "GMRES_m",
        "GMRES_GSflag", "CAGMRES_sstep", "CAGMRES_tstep", "CAGMRES_basis", "CAGMRES_QRflag",
        "CBCG_kstep", "CBCG_Eigenflag", "power_method_itrmax", "CAARNOLDI_sstep",
        "CAARNOLDI_tstep", "CAARNOLDI_basis", "CAARNOLDI_QRflag", "machineflag", "dataflag",
        "calcflag", "Neuman_itr", "Neuman_local", "itrmax")] + [
        ("rtolmax", C.c_double), ("abstolmax", C.c_double)] + [(n, C.c_int) for n in (
        "independ_nvec", "precon_thblock", "nBlock", "PRECISION_A", "PRECISION_b",
        "PRECISION_x", "PRECISION_PRECONDITION", "inner_precision", "residual_dd")] + [
        ("inner_rtol", C.c_double), ("max_refine", C.c_int), ("reserved", C.c_int * 7)]


class Crs(C.Structure):
    _fields_ = [("n", C.c_int32), ("gn", C.c_int32), ("nnz", C.c_int64), ("istart", C.c_int32),
                ("rowptr", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p)]


class Dia(C.Structure):
    _fields_ = [("n", C.c_int32), ("gn", C.c_int32), ("istart", C.c_int32), ("nnd", C.c_int32),
                ("val", C.c_void_p), ("offset", C.c_void_p)]


class Ddm(C.Structure):
    _fields_ = [("ndim", C.c_int32), ("n_grids", C.c_int32 * 3), ("margin", C.c_int32), ("m", C.c_int64),
                ("nnd", C.c_int32), ("offset", C.c_void_p), ("offset_dim", C.c_void_p), ("val", C.c_void_p),
                ("div_direc_th", C.c_int32), ("boxes", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("setup_s", C.c_double), ("solve_s", C.c_double), ("total_s", C.c_double),
                ("true_relres", C.c_double), ("true_relres_dd", C.c_double),
                ("niter", C.c_int), ("iret", C.c_int), ("refine_steps", C.c_int),
                ("kernel_launches", C.c_int), ("ilu_levels_max", C.c_int),
                ("ilu_nblocks", C.c_int), ("fallback", C.c_int), ("spmv_diagonals", C.c_int),
                ("reserved", C.c_int * 4)]


P = C.c_void_p
IP = C.POINTER(C.c_int)
I32P = C.POINTER(C.c_int32)
DP = C.POINTER(C.c_double)
PP = C.POINTER(C.c_void_p)

# DDM shim arguments after n: nnd, offset, diaA (host pointers or, _G, devicemem handles),
# num_neighbor_ranks, neighbor_ranks, margin, ndim, npe_dim, n_grids, offset_dim,
# div_direc_th, ipreflag, addL, iflagAS, niter, rtolmax, reshistory, iovlflag,
# precon_thblock, Neuman_itr, independ_nvec, nBlock (_DD: diaA_lo after diaA)
_DDM_TAIL = [IP] * 12 + [DP, P] + [IP] * 5
_DDM_H = [IP, I32P, P] + _DDM_TAIL
_DDM_G = [IP, PP, PP] + _DDM_TAIL
_DDM_DD = [IP, I32P, P, P] + _DDM_TAIL

# name -> (restype, argtypes)
SIGNATURES = {
    "parcel_init_c_": (None, [IP]),
    "parcel_free_c_": (None, []),
    "parcel_b_set_stream": (C.c_int, [P]),
    "parcel_b_get_stream": (P, []),
    "parcel_b_last_error": (C.c_int, [C.c_char_p, C.c_int]),
    "parcel_b_last_stats": (C.c_int, [C.POINTER(Stats)]),
    "parcel_b_input_init": (None, [C.POINTER(Input)]),
    "parcel_b_solve": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), P, P, P, IP, IP]),
    "parcel_dcg_c_": (None, [IP, P, P, I32P, I32P, I32P, I32P, P, P, P, IP, IP, IP, IP, IP, DP, P,
                             IP, IP, IP, IP, IP, IP]),
    "parcel_dbicgstab_c_": (None, [IP, P, P, I32P, I32P, I32P, I32P, P, P, P, IP, IP, IP, IP, IP,
                                   DP, P, IP, IP, IP, IP, IP, IP]),
    "parcel_dgmres_c_": (None, [IP, P, P, I32P, I32P, I32P, I32P, P, P, P, IP, IP, IP, IP, IP, DP,
                                P, IP, IP, IP, IP, IP, IP, IP, IP]),
    "parcel_dcagmres_c_": (None, [IP, P, P, I32P, I32P, I32P, I32P, P, P, P, IP, IP, IP, IP, IP,
                                  DP, P, IP, IP, IP, IP, IP, IP, IP, IP, IP, IP]),
    "parcel_dcg_gpu_c_": (None, [IP, PP, PP, I32P, I32P, I32P, I32P, PP, PP, PP, IP, IP, IP, IP, IP, DP,
                                 P, IP, IP, IP, IP, IP, IP]),
    "parcel_dbicgstab_gpu_c_": (None, [IP, PP, PP, I32P, I32P, I32P, I32P, PP, PP, PP, IP, IP, IP, IP,
                                       IP, DP, P, IP, IP, IP, IP, IP, IP]),
    "parcel_dgmres_gpu_c_": (None, [IP, PP, PP, I32P, I32P, I32P, I32P, PP, PP, PP, IP, IP, IP, IP, IP,
                                    DP, P, IP, IP, IP, IP, IP, IP, IP, IP]),
    "parcel_dcagmres_gpu_c_": (None, [IP, PP, PP, I32P, I32P, I32P, I32P, PP, PP, PP, IP, IP, IP, IP,
                                      IP, DP, P, IP, IP, IP, IP, IP, IP, IP, IP, IP, IP]),
    "parcel_b_setup": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), C.POINTER(P)]),
    "parcel_b_start": (C.c_int, [P, P, P, P, IP, IP]),
    "parcel_b_release": (C.c_int, [P]),
    "parcel_b_spmv": (C.c_int, [C.POINTER(Crs), P, P]),
    "parcel_b_spmv_f32": (C.c_int, [C.c_int32, C.c_int64, C.c_int32, P, P, P, P, P]),
    "parcel_b_precon_apply": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), P, P]),
    "parcel_b_dot": (C.c_int, [C.c_int64, P, P, DP]),
    "parcel_b_dot_noalloc": (C.c_int, [C.c_int64, P, P, P, P]),
    "parcel_b_residual_dd": (C.c_int, [C.POINTER(Crs), P, P, P, P, P, P]),
    "parcel_b_ddcg": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), P, C.c_int, C.c_int, C.c_int, C.c_int, P, P,
                                P, P, P, IP, IP]),
    "parcel_ddcg_c_": (None, [IP, P, P, P, P, I32P, I32P, I32P, I32P, P, P, P, P, IP, IP, IP, IP, IP, DP, P, IP,
                              IP, IP, IP, IP, IP, IP, IP, IP, IP]),
    "parcel_b_ddbicgstab": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), P, C.c_int, C.c_int, C.c_int, C.c_int, P,
                                      P, P, P, P, IP, IP]),
    "parcel_ddbicgstab_c_": (None, [IP, P, P, P, P, I32P, I32P, I32P, I32P, P, P, P, P, IP, IP, IP, IP, IP, DP, P,
                                    IP, IP, IP, IP, IP, IP, IP, IP, IP, IP]),
    "parcel_b_ddgmres": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), P, C.c_int, C.c_int, C.c_int, C.c_int, P,
                                   P, P, P, P, IP, IP]),
    "parcel_ddgmres_c_": (None, [IP, P, P, P, P, I32P, I32P, I32P, I32P, P, P, P, P, IP, IP, IP, IP, IP, DP, P,
                                 IP, IP, IP, IP, IP, IP, IP, IP, IP, IP, IP, IP]),
    "parcel_b_solve_dia": (C.c_int, [C.POINTER(Input), C.POINTER(Dia), P, P, P, IP, IP]),
    "parcel_b_ddsolve_dia": (C.c_int, [C.POINTER(Input), C.POINTER(Dia), P, C.c_int, C.c_int, C.c_int, C.c_int,
                                       P, P, P, P, P, IP, IP]),
    # DIA shims: n, gn, istart, diaA, offset, nnd in place of the CRS arguments
    "parcel_dcg_dia_c_": (None, [IP, P, P, I32P, I32P, I32P, P, P, I32P] + [IP] * 5 + [DP, P] + [IP] * 6),
    "parcel_dbicgstab_dia_c_": (None, [IP, P, P, I32P, I32P, I32P, P, P, I32P] + [IP] * 5 + [DP, P] + [IP] * 6),
    "parcel_dgmres_dia_c_": (None, [IP, P, P, I32P, I32P, I32P, P, P, I32P] + [IP] * 5 + [DP, P] + [IP] * 8),
    "parcel_dcagmres_dia_c_": (None, [IP, P, P, I32P, I32P, I32P, P, P, I32P] + [IP] * 5 + [DP, P] + [IP] * 10),
    "parcel_dcg_dia_gpu_c_": (None, [IP, P, P, I32P, I32P, I32P, P, P, I32P] + [IP] * 5 + [DP, P] + [IP] * 6),
    "parcel_dbicgstab_dia_gpu_c_": (None, [IP, P, P, I32P, I32P, I32P, P, P, I32P] + [IP] * 5 + [DP, P] +
                                    [IP] * 6),
    "parcel_dgmres_dia_gpu_c_": (None, [IP, P, P, I32P, I32P, I32P, P, P, I32P] + [IP] * 5 + [DP, P] + [IP] * 8),
    "parcel_dcagmres_dia_gpu_c_": (None, [IP, P, P, I32P, I32P, I32P, P, P, I32P] + [IP] * 5 + [DP, P] +
                                   [IP] * 10),
    "parcel_ddcg_dia_c_": (None, [IP, P, P, P, P, I32P, I32P, I32P, P, P, P, I32P] + [IP] * 5 + [DP, P] +
                           [IP] * 10),
    "parcel_ddbicgstab_dia_c_": (None, [IP, P, P, P, P, I32P, I32P, I32P, P, P, P, I32P] + [IP] * 5 + [DP, P] +
                                 [IP] * 10),
    "parcel_ddgmres_dia_c_": (None, [IP, P, P, P, P, I32P, I32P, I32P, P, P, P, I32P] + [IP] * 5 + [DP, P] +
                              [IP] * 11),
    "parcel_b_solve_ddm": (C.c_int, [C.POINTER(Input), C.POINTER(Ddm), P, P, P, IP, IP]),
    "parcel_b_ddsolve_ddm": (C.c_int, [C.POINTER(Input), C.POINTER(Ddm), P, C.c_int, C.c_int, C.c_int, C.c_int,
                                       P, P, P, P, P, IP, IP]),
    "parcel_b_ddm_order": (C.c_int, [C.POINTER(Ddm), C.c_int, I32P, I32P, I32P]),
    "parcel_b_bench_kernels_ddm": (C.c_int, [C.POINTER(Input), C.POINTER(Ddm), C.c_int, DP, DP]),
    # DDM shims: n (padded cells), nnd, offset, diaA, the decomposition and the solver arguments
    "parcel_dcg_ddm_c_": (None, [IP, P, P, I32P] + _DDM_H + [IP]),
    "parcel_dbicgstab_ddm_c_": (None, [IP, P, P, I32P] + _DDM_H + [IP]),
    "parcel_dgmres_ddm_c_": (None, [IP, P, P, I32P] + _DDM_H + [IP] * 3),
    "parcel_dcagmres_ddm_c_": (None, [IP, P, P, I32P] + _DDM_H + [IP] * 5),
    "parcel_ddcg_ddm_c_": (None, [IP, P, P, P, P, I32P] + _DDM_DD + [IP] * 5),
    "parcel_ddbicgstab_ddm_c_": (None, [IP, P, P, P, P, I32P] + _DDM_DD + [IP] * 5),
    "parcel_ddgmres_ddm_c_": (None, [IP, P, P, P, P, I32P] + _DDM_DD + [IP] * 7),
    "parcel_dcg_ddm_gpu_c_": (None, [IP, PP, PP, I32P] + _DDM_G + [IP]),
    "parcel_dbicgstab_ddm_gpu_c_": (None, [IP, PP, PP, I32P] + _DDM_G + [IP]),
    "parcel_dgmres_ddm_gpu_c_": (None, [IP, PP, PP, I32P] + _DDM_G + [IP] * 3),
    "parcel_dcagmres_ddm_gpu_c_": (None, [IP, PP, PP, I32P] + _DDM_G + [IP] * 5),
    "parcel_b_local_create_blocks": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), C.c_int, C.c_int, I32P,
                                               C.POINTER(P)]),
    "parcel_b_bench_kernels": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), C.c_int, DP, DP]),
    "parcel_b_local_create": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), C.c_int, C.POINTER(P)]),
    "parcel_b_local_spmv": (C.c_int, [P, P, P]),
    "parcel_b_local_precon": (C.c_int, [P, P, P]),
    "parcel_b_local_destroy": (C.c_int, [P]),
    "parcel_b_learned_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(P)]),
    "parcel_b_learned_destroy": (C.c_int, [P]),
    "parcel_b_learned_num_params": (C.c_int64, []),
    "parcel_b_learned_get_params": (C.c_int, [P, P, DP]),
    "parcel_b_learned_set_params": (C.c_int, [P, P, C.c_double]),
    "parcel_b_learned_forward": (C.c_int, [P, C.c_int, P, P]),
    "parcel_b_learned_grad": (C.c_int, [P, C.c_int, P, P, DP, P]),
    "parcel_b_learned_adam": (C.c_int, [P, C.c_double]),
    "parcel_b_learned_collect": (C.c_int, [P, C.POINTER(Input), C.POINTER(Crs), P, C.c_int, IP]),
    "parcel_b_learned_num_pairs": (C.c_int, [P]),
    "parcel_b_learned_train": (C.c_int, [P, C.c_int, C.c_int, C.c_double, C.c_uint64, DP, DP]),
    "parcel_b_learned_set_stage": (C.c_int, [P, C.c_int, C.c_int]),
    "parcel_b_learned_galerkin": (C.c_int, [P, C.POINTER(Crs), P]),
    "parcel_b_learned_coarse_solve": (C.c_int, [P, C.POINTER(Crs), P, P, C.c_int, P]),
    "parcel_b_learned_transfer": (C.c_int, [P, C.c_int, P, P]),
    "parcel_b_solve_learned": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), P, P, P, P, IP, IP]),
    "parcel_b_solve_learned_many": (C.c_int, [C.POINTER(Input), C.POINTER(Crs), P, C.c_int, P, P, P, P]),
}

_lib = None


def load() -> C.CDLL:
    """Loads libparcelb.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with python parcel-legacy_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(512)
    code = load().parcel_b_last_error(buf, 512)
    return f"[{code}] {buf.value.decode(errors='replace')}"


def last_stats() -> dict:
    s = Stats()
    load().parcel_b_last_stats(C.byref(s))
    return {k: getattr(s, k) for k, _ in Stats._fields_ if k != "reserved"}


def new_input(**kw) -> Input:
    p = Input()
    load().parcel_b_input_init(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p
