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


def test_ddm_struct_layout_matches_c(tmp_path):
    src = tmp_path / "ddm.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "parcel_b.h"\n'
                   'int main(){printf("%zu %zu %zu %zu %zu\\n", sizeof(parcel_b_ddm), offsetof(parcel_b_ddm, m), '
                   'offsetof(parcel_b_ddm, offset), offsetof(parcel_b_ddm, val), offsetof(parcel_b_ddm, boxes));'
                   'return 0;}\n')
    exe = tmp_path / "ddm"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    D = _lib.Ddm
    assert [int(v) for v in out] == [C.sizeof(D), D.m.offset, D.offset.offset, D.val.offset, D.boxes.offset]


def test_ddm_shim_signatures_count_the_reference_arguments():
    """parcel_dcg_ddm_c takes 27 arguments (c2fortran_kernel.f90:2964-2983), the dd form 34
    (3272-3295)."""
    decl = _c_declarations()
    assert len(decl["parcel_dcg_ddm_c_"][1]) == 27 == len(_lib.SIGNATURES["parcel_dcg_ddm_c_"][1])
    assert len(decl["parcel_dgmres_ddm_c_"][1]) == 29 == len(_lib.SIGNATURES["parcel_dgmres_ddm_c_"][1])
    assert len(decl["parcel_ddcg_ddm_c_"][1]) == 34 == len(_lib.SIGNATURES["parcel_ddcg_ddm_c_"][1])
    assert len(decl["parcel_dcagmres_ddm_gpu_c_"][1]) == 31 == len(_lib.SIGNATURES["parcel_dcagmres_ddm_gpu_c_"][1])


def test_input_defaults_are_minus_one():
    p = _lib.new_input()
    for f in ("ipreflag", "ILU_method", "solver", "GMRES_m", "itrmax", "precon_thblock", "independ_nvec"):
        assert getattr(p, f) == -1
    assert p.rtolmax == -1.0


FORTRAN = os.path.join(ROOT, "parcel-legacy_b200", "fortran", "parcel_b_iso.f90")


def _fortran_source():
    src = re.sub(r"!.*", "", open(FORTRAN).read())
    return re.sub(r"&\s*\n\s*", " ", src)


def _c_declarations():
    hdr = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(void|int)\s+(parcel_\w+)\s*\(([^)]*)\)", hdr):
        args = [a.strip() for a in m.group(3).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(2)] = (m.group(1), args)
    return out


def _fortran_kind(c_arg):
    """The Fortran declaration a C parameter must have in a bind(c) interface (the name is
    dropped, so only the type and the pointer level remain)."""
    t = re.sub(r"\bconst\b", "", c_arg)
    t = re.sub(r"\w+$", "", t.strip()).replace(" ", "")
    return {"double*": {"real(c_double)", "type(c_ptr),value"}, "int32_t*": {"integer(c_int32_t)"},
            "int*": {"integer(c_int)"}, "int": {"integer(c_int),value"}, "void**": {"type(c_ptr)"},
            "parcel_b_input*": {"type(KSP_INPUT_PARAM)"}, "parcel_b_crs*": {"type(parcel_b_crs_t)"}}[t]


def test_fortran_interfaces_match_the_header():
    """parcel_b_iso.f90 is shipped uncompiled (no Fortran compiler in this image): check that
    each bind(c) interface (subroutine or integer function) has the C declaration's
    arguments, in order, with matching kinds and passing (by value or by reference)."""
    decls = _c_declarations()
    src = _fortran_source()
    stmts = re.findall(r"(subroutine|integer\(c_int\) function)\s+(c_\w+)\s*\(([^)]*)\)\s*bind\(c,\s*name=\"(\w+)\"\)",
                       src)
    stmts += [("subroutine", n, "", s) for n, s in
              re.findall(r"subroutine\s+(c_\w+)\s*\(\)\s*bind\(c,\s*name=\"(\w+)\"\)", src)]
    assert len(stmts) >= 26
    for kind, name, args, sym in stmts:
        fargs = [a.strip().lower() for a in args.split(",") if a.strip()]
        end = "end subroutine" if kind == "subroutine" else "end function"
        body = re.search(r"%s\s*\(.*?%s %s" % (name, end, name), src, flags=re.S).group(0)
        kinds = {}
        for decl, names in re.findall(r"(integer\(c_int\)(?:,\s*value)?|integer\(c_int32_t\)|real\(c_double\)|"
                                      r"type\(c_ptr\)(?:,\s*value)?|type\(KSP_INPUT_PARAM\)|type\(parcel_b_crs_t\))"
                                      r"\s*::\s*([^\n]*)", body):
            for nm in names.split(","):
                kinds[re.sub(r"\(\*\)", "", nm.strip()).lower()] = decl.replace(" ", "")
        assert sym in decls, sym
        ret, cargs = decls[sym]
        assert (ret == "void") == (kind == "subroutine"), sym
        assert len(cargs) == len(fargs), sym
        for ca, fa in zip(cargs, fargs):
            assert kinds.get(fa) in _fortran_kind(ca), (sym, ca, fa, kinds.get(fa))


def _c_struct_fields(name):
    hdr = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), hdr, flags=re.S).group(1)
    out = []
    for decl in body.split(";"):
        decl = decl.replace("const", " ").strip()
        if not decl:
            continue
        m = re.match(r"(\w+\s*\**)\s*(.+)$", decl)
        t, names = m.group(1).replace(" ", ""), m.group(2)
        for nm in names.split(","):
            nm = nm.strip()
            n_ = int(re.search(r"\[(\d+)\]", nm).group(1)) if "[" in nm else 1
            out.append((re.sub(r"\[.*", "", nm), t.replace("const", "").strip(), n_))
    return out


def _f_type_fields(name):
    src = _fortran_source()
    body = re.search(r"type,\s*bind\(c\)\s*::\s*%s(.*?)end type %s" % (name, name), src, flags=re.S).group(1)
    out = []
    for t, names in re.findall(r"(integer\(c_int\)|integer\(c_int32_t\)|integer\(c_int64_t\)|real\(c_double\)|"
                               r"type\(c_ptr\))\s*::\s*([^\n]*)", body):
        for nm in names.split(","):
            nm = nm.strip()
            n_ = int(re.search(r"\((\d+)\)", nm).group(1)) if "(" in nm else 1
            out.append((re.sub(r"\(.*", "", nm), t, n_))
    return out


def test_fortran_types_match_the_c_structs():
    """type(KSP_INPUT_PARAM) of module krylov is parcel_b_input member for member (names,
    order, kinds, array lengths), and parcel_b_crs_t is parcel_b_crs, so C's and Fortran's
    layout rules give both the same offsets."""
    ckind = {"int": "integer(c_int)", "int32_t": "integer(c_int32_t)", "int64_t": "integer(c_int64_t)",
             "double": "real(c_double)", "int32_t*": "type(c_ptr)", "double*": "type(c_ptr)"}
    for cname, fname in (("parcel_b_input", "KSP_INPUT_PARAM"), ("parcel_b_crs", "parcel_b_crs_t")):
        c = [(n.lower(), ckind[t.replace(" ", "")], k) for n, t, k in _c_struct_fields(cname)]
        f = [(n.lower(), t, k) for n, t, k in _f_type_fields(fname)]
        assert c == f, (cname, c, f)
    # the reference's KSP_INPUT_PARAM fields come first, in the reference's order
    # (src/type.f90:907-946)
    ref = ["ipreflag", "ilu_method", "addl", "iflagas", "solver", "iovlflag", "gmres_m", "gmres_gsflag",
           "cagmres_sstep", "cagmres_tstep", "cagmres_basis", "cagmres_qrflag", "cbcg_kstep", "cbcg_eigenflag",
           "power_method_itrmax", "caarnoldi_sstep", "caarnoldi_tstep", "caarnoldi_basis", "caarnoldi_qrflag",
           "machineflag", "dataflag", "calcflag", "neuman_itr", "neuman_local", "itrmax", "rtolmax", "abstolmax",
           "independ_nvec", "precon_thblock", "nblock", "precision_a", "precision_b", "precision_x",
           "precision_precondition"]
    assert [n.lower() for n, _, _ in _f_type_fields("KSP_INPUT_PARAM")][:len(ref)] == ref


def test_fortran_wrapper_provides_the_reference_entry_points():
    """Module PARCEL_wrapper offers the reference's generic entries and both builds' forms of
    the solver wrappers (host arrays, or device addresses as type(c_ptr))."""
    src = _fortran_source().lower()
    for name in ("init_parcel_input", "parcel_ddksp_crs", "parcel_dcg_host", "parcel_dcg_dev", "parcel_dgmres_dev",
                 "parcel_dbicgstab_dev", "parcel_dcagmres_dev", "parcel_ksp_crs_host", "parcel_ksp_crs_dev"):
        assert re.search(r"subroutine %s\s*\(" % name, src), name
    for generic in ("parcel_ksp_crs", "parcel_dcg", "parcel_dbicgstab", "parcel_dgmres", "parcel_dcagmres"):
        m = re.search(r"interface %s\s+module procedure ([\w, ]+)" % generic, src)
        assert m and {generic + "_host", generic + "_dev"} == {p.strip() for p in m.group(1).split(",")}, generic
    for mod in ("parcel_integer", "parcel_define", "krylov", "parcel_wrapper"):
        assert re.search(r"^module %s\b" % mod, src, flags=re.M), mod


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


def test_fortran_ddm_wrapper_module_exports_the_reference_names():
    """src/example/main_ddm.f90 uses module ddm_wrapper's parcel_d*_ddm routines."""
    src = _fortran_source()
    m = re.search(r"module ddm_wrapper(.*?)end module ddm_wrapper", src, flags=re.S)
    assert m
    public = re.search(r"public\s*::\s*([^\n]*)", m.group(1)).group(1)
    names = {n.strip() for n in public.split(",")}
    assert names == {"parcel_dcg_ddm", "parcel_dbicgstab_ddm", "parcel_dgmres_ddm", "parcel_dcagmres_ddm",
                     "parcel_ddcg_ddm", "parcel_ddbicgstab_ddm", "parcel_ddgmres_ddm"}
    for n in names:
        assert re.search(r"subroutine %s\s*\(" % n, m.group(1)) and re.search(r"call c_%s\s*\(" % n, m.group(1))
