"""The host eigen-solvers of the direct Poisson solve (moons_b200/csrc/eig.hpp:
implicit QL on tridiagonal matrices, Householder reduction + QL and cyclic
Jacobi on full ones), compiled for the host with g++ and checked against
numpy: A V = V diag(w), V orthonormal, eigenvalues as numpy's."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <cstdio>
#include "eig.hpp"
int main() {
  int mode, n;
  if (scanf("%d %d", &mode, &n) != 2) return 1;
  std::vector<double> A((size_t)n * n);
  for (auto& v : A) if (scanf("%lf", &v) != 1) return 1;
  std::vector<double> w, V;
  if (mode == 0) {
    std::vector<double> d(n), e(n, 0.0);
    for (int i = 0; i < n; i++) d[i] = A[(size_t)i * n + i];
    for (int i = 0; i + 1 < n; i++) e[i] = A[(size_t)i * n + i + 1];
    if (!eig::tridiag_ql(d, e, n, w, V)) return 2;
  } else if (mode == 1) {
    eig::symmetric_eigen(A, n, w, V);
  } else {
    eig::jacobi_eigen(A, n, w, V);
  }
  for (double x : w) printf("%.17g\n", x);
  for (double x : V) printf("%.17g\n", x);
  return 0;
}
"""


@pytest.fixture(scope="module")
def exe():
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    d = os.path.join(ROOT, "tests", "_build")
    os.makedirs(d, exist_ok=True)
    src = os.path.join(d, "eig_harness.cpp")
    out = os.path.join(d, "eig_harness")
    with open(src, "w") as f:
        f.write(HARNESS)
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "moons_b200", "csrc"), "-o", out, src],
                   check=True, capture_output=True)
    return out


def run(exe, mode, A):
    n = A.shape[0]
    inp = f"{mode} {n}\n" + " ".join(repr(float(x)) for x in A.ravel())
    r = subprocess.run([exe], input=inp, capture_output=True, text=True)
    assert r.returncode == 0, r.returncode
    v = np.array(r.stdout.split(), dtype=float)
    return v[:n], v[n:].reshape(n, n)


def check(A, w, V):
    n = A.shape[0]
    scale = max(np.abs(A).max(), 1e-300)
    assert np.abs(A @ V - V * w[None, :]).max() <= 1e-12 * scale * max(1, n / 64)
    assert np.abs(V.T @ V - np.eye(n)).max() <= 1e-12 * max(1, n / 64)
    assert np.abs(np.sort(w) - np.linalg.eigvalsh(A)).max() <= 1e-11 * scale * max(1, n / 64)


@pytest.mark.parametrize("n", [1, 2, 3, 10, 65, 200])
def test_tridiagonal_ql(exe, n):
    rng = np.random.default_rng(n)
    d, e = rng.standard_normal(n) * 3, rng.standard_normal(max(n - 1, 0))
    if n > 8:
        e[n // 3] = 0.0   # a block that splits
    A = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    check(A, *run(exe, 0, A))


@pytest.mark.parametrize("mode", [1, 2], ids=["householder_ql", "jacobi"])
@pytest.mark.parametrize("n", [1, 2, 5, 33, 96])
def test_full_symmetric(exe, mode, n):
    rng = np.random.default_rng(100 + n)
    A = rng.standard_normal((n, n))
    check(A + A.T, *run(exe, mode, A + A.T))


@pytest.mark.parametrize("n", [4, 5, 64, 256])
def test_cyclic_second_difference(exe, n):
    # a periodic axis: degenerate pairs and the zero (constant) mode
    A = np.zeros((n, n))
    for i in range(n):
        A[i, i] = -2.0
        A[i, (i + 1) % n] = A[(i + 1) % n, i] = 1.0
    A *= 1024.0
    w, V = run(exe, 1, A)
    check(A, w, V)
    z = int(np.argmin(np.abs(w)))
    assert abs(w[z]) < 1e-9 * np.abs(w).max()
    assert np.allclose(np.abs(V[:, z]), 1.0 / np.sqrt(n))
