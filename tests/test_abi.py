"""CPU-side checks of the C-ABI: the library loads and exports every function that
include/parcel_b.h declares, and the ctypes mirrors of its structs have the C layout."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT
from parcel_b import _lib

HEADER = os.path.join(ROOT, "include", "parcel_b.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:[\w\*]+\s+)+\**(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n.startswith(("parcel", "PARCEL"))))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for n in ("parcel_dcg_c_", "parcel_dbicgstab_c_", "parcel_dgmres_c_", "parcel_dcagmres_c_",
              "parcel_init_c_", "parcel_free_c_", "parcel_b_solve", "parcel_ddcg_c_", "parcel_ddbicgstab_c_",
              "parcel_ddgmres_c_", "parcel_dcg_dia_c_", "parcel_dbicgstab_dia_c_", "parcel_dgmres_dia_c_",
              "parcel_dcagmres_dia_c_", "parcel_ddcg_dia_c_", "parcel_ddbicgstab_dia_c_", "parcel_ddgmres_dia_c_"):
        assert n in names


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_the_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "parcel_b.h"\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(parcel_b_input), '
                   'sizeof(parcel_b_stats), sizeof(parcel_b_crs), offsetof(parcel_b_input, rtolmax), '
                   'offsetof(parcel_b_input, inner_rtol), offsetof(parcel_b_crs, rowptr), '
                   'sizeof(parcel_b_dia), offsetof(parcel_b_dia, offset));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    want = [C.sizeof(_lib.Input), C.sizeof(_lib.Stats), C.sizeof(_lib.Crs), _lib.Input.rtolmax.offset,
            _lib.Input.inner_rtol.offset, _lib.Crs.rowptr.offset, C.sizeof(_lib.Dia), _lib.Dia.offset.offset]
    assert [int(v) for v in out] == want


def test_input_defaults_are_minus_one():
    p = _lib.new_input()
    for f in ("ipreflag", "ILU_method", "solver", "GMRES_m", "itrmax", "precon_thblock", "independ_nvec"):
        assert getattr(p, f) == -1
    assert p.rtolmax == -1.0


def test_fortran_interfaces_match_the_header():
    """parcel_b_iso.f90 is shipped uncompiled (no Fortran compiler in this image): check that
    each bind(c) interface has the C declaration's arguments, in order, with matching kinds."""
    hdr = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    decls = {m.group(1): [a.strip() for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
             for m in re.finditer(r"void\s+(parcel_\w+_c_)\s*\(([^)]*)\)", hdr)}
    src = open(os.path.join(ROOT, "parcel-legacy_b200", "fortran", "parcel_b_iso.f90")).read()
    src = re.sub(r"&\s*\n\s*", " ", src)
    stmts = re.findall(r"subroutine\s+(c_\w+)\s*\(([^)]*)\)\s*bind\(c,\s*name=\"(\w+)\"\)", src)
    stmts += [(n, "", s) for n, s in re.findall(r"subroutine\s+(c_\w+)\s*\(\)\s*bind\(c,\s*name=\"(\w+)\"\)", src)]
    assert len(stmts) >= 16
    for name, args, sym in stmts:
        fargs = [a.strip() for a in args.split(",") if a.strip()]
        body = re.search(r"subroutine\s+%s\s*\(.*?end subroutine %s" % (name, name), src, flags=re.S).group(0)
        kinds = {}
        for kind, names in re.findall(r"(integer\(c_int\)|integer\(c_int32_t\)|real\(c_double\))\s*::\s*([^\n]*)",
                                      body):
            for nm in names.split(","):
                kinds[re.sub(r"\(\*\)", "", nm.strip()).lower()] = kind
        assert sym in decls, sym
        assert len(decls[sym]) == len(fargs), sym
        for ca, fa in zip(decls[sym], fargs):
            ct = ca.replace(" ", "")
            want = ("real(c_double)" if ct.startswith("double*") else
                    "integer(c_int32_t)" if ct.startswith("int32_t*") else "integer(c_int)")
            assert kinds.get(fa.lower()) == want, (sym, ca, fa, kinds.get(fa.lower()))


def test_python_api_rejects_mistyped_arrays_before_calling_the_library():
    """Wrong element types or lengths raise in Python; nothing reaches the C side."""
    import numpy as np
    from parcel_b import api, problems
    A = problems.convdiff3d_upwind(4)
    b = np.ones(A.n)
    val = np.zeros(7 * A.n)
    off = np.array([-16, -4, -1, 0, 1, 4, 16], dtype=np.int32)
    with pytest.raises(TypeError, match="offset must be int32"):
        api.solve_dia(val, off.astype(np.int64), b)
    with pytest.raises(ValueError, match="val has"):
        api.solve_dia(val[:-1], off, b)
    with pytest.raises(TypeError, match="b must be float64"):
        api.solve_dia(val, off, b.astype(np.float32))
    with pytest.raises(ValueError, match="val_lo has"):
        api.ddsolve_dia(val, off, b, val_lo=np.zeros(3))
    with pytest.raises(ValueError, match="val_lo has"):
        api.ddcg(A, b, val_lo=np.zeros(A.nnz + 1))
    with pytest.raises(TypeError, match="b_lo must be float64"):
        api.ddgmres(A, b, b_lo=np.zeros(A.n, dtype=np.float32))
