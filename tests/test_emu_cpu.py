"""CPU emulation of the fused PCG kernels' point math against the oracle.

The __host__ __device__ point functions of moons_b200/csrc/fused.cuh are
compiled into a host program with nvcc and compared point by point with the
oracle's apply_BCs_implicit -> operator -> masks -> vol sequence for every
PCG operator and a set of BC mixes (periodic, Robin, per-component)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not available")
def test_fused_point_math_matches_oracle():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    out = os.path.join(ROOT, "tests", "_build", "emu_fused")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run([nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-o", out,
                    os.path.join(ROOT, "tests", "emu", "emu_fused.cu"), os.path.join(ROOT, "oracle", "moons_oracle.cpp")],
                   check=True, capture_output=True)
    r = subprocess.run([out], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-3000:]
    assert "ALL OK" in r.stdout


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not available")
def test_time_scheme_point_math_matches_oracle():
    """scheme_increment / scheme_rhs (moons_b200/csrc/schemes.cuh), the point
    arithmetic k_ab2_rhs runs for every time scheme, bit for bit against the
    reference's whole-array sequences on the oracle's primitives."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    out = os.path.join(ROOT, "tests", "_build", "emu_schemes")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run([nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-o", out,
                    os.path.join(ROOT, "tests", "emu", "emu_schemes.cu"), os.path.join(ROOT, "oracle", "moons_oracle.cpp")],
                   check=True, capture_output=True)
    r = subprocess.run([out], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-3000:]
    assert "ALL OK" in r.stdout
