"""Extracts the reference's stored example outputs into small JSON fixtures.

Run once in a checkout that has the reference mounted (it reads the reference's text
output files; nothing here executes reference code):

    python tests/golden/make_golden.py <path of the reference checkout>

Writes tests/golden/reference_templates.json.  The fixtures are the reference's only
known-answer outputs for this path (src/example/template_cpu/STDOUT_run,
template_gpu/STDOUT_run, template_cpu/STDOUT_run_dd, template_cpu/STDOUT_run_qr, and the
DDM ones template_cpu/STDOUT_run_ddm, template_gpu/STDOUT_run_ddm,
template_cpu/STDOUT_run_ddm_dd), all for the 160^3 Poisson problem of the examples with
rtolmax = 1e-9.
"""
from __future__ import annotations

import json
import os
import re
import sys


def parse_history(path: str):
    crs, other = [], []
    for line in open(path):
        m = re.match(r"\s*PARCEL : @res@\s+(\d+)\s+(\S+)\s+(\S+)", line)
        if m:
            crs.append(float(m.group(2).replace("D", "E")))
            other.append(float(m.group(3).replace("D", "E")))
    return crs, other


def parse_errors(path: str):
    out = {}
    for line in open(path):
        if "max(|numerical-exact|) / max(|exact|)" in line:
            out["rel_err"] = float(line.split("=")[-1])
        elif "max(|numerical-exact|)" in line:
            out["abs_err"] = float(line.split("=")[-1])
    return out


def parse_ddm_history(path: str):
    """main_ddm.f90 prints `i reshistory(i)` for the iterations used, then the timings."""
    h = []
    for line in open(path):
        m = re.match(r"\s*(\d+)\s+(\S+)\s*$", line)
        if m:
            h.append(float(m.group(2).replace("D", "E")))
    return h


def parse_qr(path: str):
    return [line.rstrip("\n") for line in open(path)]


def main(ref: str) -> None:
    ex = os.path.join(ref, "src", "example")
    fx = {}
    crs, dia = parse_history(os.path.join(ex, "template_cpu", "STDOUT_run"))
    fx["cpu_cg_dilu80"] = {
        "source": "src/example/template_cpu/STDOUT_run",
        "problem": "make_poisson3D_CRS 160x160x160, RHS make_poisson3D_right_vector, x0 = 0",
        "solver": "CG", "ipreflag": 2, "ILU_method": 1, "blocks": 80,
        "blocks_note": "4 MPI ranks x 20 OpenMP threads -> 80 contiguous blocks of 51,200 rows",
        "rtolmax": 1e-9, "history_crs": crs, "history_dia": dia,
        **parse_errors(os.path.join(ex, "template_cpu", "STDOUT_run")),
    }
    crs, dia = parse_history(os.path.join(ex, "template_gpu", "STDOUT_run"))
    fx["gpu_cg_ilu0_4"] = {
        "source": "src/example/template_gpu/STDOUT_run",
        "problem": "make_poisson3D_CRS 160x160x160, RHS make_poisson3D_right_vector, x0 = 0",
        "solver": "CG", "ipreflag": 2, "ILU_method": "ignored on GPU: cuSPARSE ILU(0)",
        "blocks": 4, "blocks_note": "4 MPI ranks, one cuSPARSE ILU(0) block per rank",
        "rtolmax": 1e-9, "history_crs": crs, "history_dia": dia,
        **parse_errors(os.path.join(ex, "template_gpu", "STDOUT_run")),
    }
    dd, dbl = parse_history(os.path.join(ex, "template_cpu", "STDOUT_run_dd"))
    half = len(dd) // 2 if len(dd) > 400 else len(dd)
    fx["cpu_cg_dilu80_dd"] = {
        "source": "src/example/template_cpu/STDOUT_run_dd",
        "history_dd": dd[:half], "history_double": dbl[:half],
        **parse_errors(os.path.join(ex, "template_cpu", "STDOUT_run_dd")),
    }
    ddm = "make_poisson_3D_DDM 160x160x160 on npe = (1, 4, 1), RHS of the example, x0 = 0"
    fx["cpu_ddm_cg_slabs"] = {
        "source": "src/example/template_cpu/STDOUT_run_ddm", "problem": ddm, "solver": "CG", "ipreflag": 2,
        "npe": [1, 4, 1], "div_direc_th": 1, "threads": 20,
        "blocks_note": "4 processes x 20 OpenMP threads: D-ILU on 80 boxes of 8 x 40 x 160 cells",
        "rtolmax": 1e-9, "history": parse_ddm_history(os.path.join(ex, "template_cpu", "STDOUT_run_ddm")),
    }
    fx["gpu_ddm_cg_cubes"] = {
        "source": "src/example/template_gpu/STDOUT_run_ddm", "problem": ddm, "solver": "CG", "ipreflag": 2,
        "npe": [1, 4, 1], "blocks_note": "CUDA build (DDM_CUDA_BJ): D-ILU on 4 x 4 x 4 boxes",
        "rtolmax": 1e-9, "history": parse_ddm_history(os.path.join(ex, "template_gpu", "STDOUT_run_ddm")),
    }
    fx["cpu_ddm_ddcg_slabs"] = {
        "source": "src/example/template_cpu/STDOUT_run_ddm_dd", "problem": ddm, "solver": "ddCG", "ipreflag": 2,
        "npe": [1, 4, 1], "div_direc_th": 1, "threads": 20, "precision": [2, 2, 2, 2],
        "rtolmax": 1e-9, "history": parse_ddm_history(os.path.join(ex, "template_cpu", "STDOUT_run_ddm_dd")),
    }
    fx["cpu_qr"] = {"source": "src/example/template_cpu/STDOUT_run_qr",
                    "lines": parse_qr(os.path.join(ex, "template_cpu", "STDOUT_run_qr"))}
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_templates.json")
    with open(out, "w") as f:
        json.dump(fx, f, indent=1)
    print("wrote", out, {k: len(v.get("history_crs", v.get("history_dd", v.get("history", [])))) for k, v in fx.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
