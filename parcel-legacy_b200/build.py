"""Build recipe of libparcelb.so (sm_100a) -- the product library.

    python parcel-legacy_b200/build.py [-j N] [--debug]

Compiles every csrc/*.cu with nvcc for sm_100a into parcel-legacy_b200/libparcelb.so
(in-tree, so it travels with the repository to the GPU host).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libparcelb.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def flags(debug: bool):
    f = ARCH + ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", "-ccbin", "/usr/bin/g++",
                "-I", os.path.join(HERE, "..", "include"), "--expt-relaxed-constexpr", "-Xptxas", "-v" if debug else "-O3"]
    return f


def compile_one(src: str, debug: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    deps = glob.glob(os.path.join(CSRC, "*.cuh")) + [src, os.path.join(HERE, "..", "include", "parcel_b.h")]
    if os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [NVCC] + flags(debug) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise SystemExit(f"nvcc failed on {src}")
    if debug:
        sys.stderr.write(r.stderr)
    return obj


def build(jobs: int = 8, debug: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: compile_one(s, debug), srcs))
    cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC,-fopenmp", "-ccbin", "/usr/bin/g++", "-o", LIB] + objs + ["-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise SystemExit("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--debug", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.debug))
