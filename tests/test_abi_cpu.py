"""The C-ABI library loads without a GPU and exports every function that
include/moons_gpu.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "moons_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(moons_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for n in ("moons_mesh_create", "moons_sf_upload", "moons_apply_bcs", "moons_pcg_create", "moons_pcg_solve",
              "moons_mhd_step", "moons_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from moons_b200 import build
    if build.needs_build():
        build.build()
    lib = ctypes.CDLL(build.LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_last_error_without_gpu():
    from moons_b200 import build
    lib = ctypes.CDLL(build.LIB)
    lib.moons_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.moons_last_error(), bytes)


def _c_layout(structs):
    """sizeof and field offsets of the header's structs, as the C compiler
    lays them out (gcc on a small program that includes the header)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("gcc not available")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "moons_gpu.h"', "int main(void) {"]
    for cname, fields in structs:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    d = os.path.join(ROOT, "tests", "_build")
    os.makedirs(d, exist_ok=True)
    src, exe = os.path.join(d, "abi_layout.c"), os.path.join(d, "abi_layout")
    with open(src, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            parts = ln.split()
            got[(parts[0], parts[1])] = int(parts[2])
    return got


def test_ctypes_structs_match_the_header_layout():
    """The ctypes mirrors of the parameter and report structs (moons_b200.capi,
    also used by the oracle's bindings) have the C sizes and field offsets."""
    from moons_b200 import capi as G
    mirrors = [("moons_bc_spec", G.BCSpec), ("moons_isp", G.ISP), ("moons_solve_info", G.SolveInfo),
               ("moons_mhd_params", G.MHDParams), ("moons_step_info", G.StepInfo)]
    got = _c_layout([(c, [f for f, _ in py._fields_]) for c, py in mirrors])
    for cname, py in mirrors:
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


FORTRAN = os.path.join(ROOT, "fortran", "moons_gpu_mod.f90")


def _header_functions():
    """{name: number of parameters} of the header's function declarations."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(moons_[a-z0-9_]+)\s*\(([^()]*)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else len(params.split(","))
    return out


def _fortran_text():
    text = open(FORTRAN).read()
    text = re.sub(r"!.*", "", text)                 # comments
    return re.sub(r"&\s*\n\s*&?", " ", text)          # continuation lines


def test_fortran_bindings_match_the_header():
    """Every bind(C) interface of the Fortran module names a function the
    header declares, with the same number of arguments."""
    decl = _header_functions()
    bound = re.findall(r"function\s+\w+\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", _fortran_text(), flags=re.I)
    assert len(bound) >= 20
    for args, name in bound:
        assert name in decl, name
        n = 0 if not args.strip() else len(args.split(","))
        assert n == decl[name], (name, n, decl[name])


def test_fortran_types_match_the_header_structs():
    """The module's bind(C) derived types list the C structs' fields in the
    same order, with the same names and array extents, so their layouts
    agree."""
    ftext = _fortran_text()
    ctext = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    for tname in ("moons_bc_spec", "moons_isp", "moons_solve_info", "moons_mhd_params", "moons_step_info"):
        m = re.search(r"type,\s*bind\(C\)\s*::\s*" + tname + r"(.*?)end type", ftext, flags=re.S | re.I)
        assert m, tname
        ffields = []
        for line in m.group(1).strip().splitlines():
            names = line.split("::")[1]
            ffields += [x.strip().replace("(", "[").replace(")", "]") for x in names.split(",")]
        c = re.search(r"typedef struct \{([^{}]*)\}\s*" + tname + r"\s*;", ctext)
        assert c, tname
        cfields = []
        for decl in c.group(1).split(";"):
            decl = decl.strip()
            if decl:
                rest = decl.split(None, 1)[1]
                cfields += [x.strip(" *") for x in rest.split(",")]
        assert ffields == cfields, (tname, ffields, cfields)


def test_ctypes_bindings_match_the_header():
    """moons_b200/capi.py declares every header function, with the header's
    number of arguments (its signature table, read without loading it)."""
    import ast
    tree = ast.parse(open(os.path.join(ROOT, "moons_b200", "capi.py")).read())
    table = None
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Dict) and \
                any(isinstance(t, ast.Name) and t.id == "sig" for t in node.targets):
            table = node.value
    assert table is not None
    decl = _header_functions()
    names = []
    for k, v in zip(table.keys, table.values):
        name, nargs = k.value, len(v.elts[1].elts)
        names.append(name)
        assert name in decl, name
        assert nargs == decl[name], (name, nargs, decl[name])
    assert sorted(names) == sorted(decl)
