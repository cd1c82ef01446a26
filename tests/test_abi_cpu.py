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
