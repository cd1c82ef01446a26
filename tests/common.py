"""Shared helpers of the test-suite: meshes, seeded fields and the
side-by-side driver of the product (moons_b200.capi) and the oracle."""
from __future__ import annotations

import numpy as np

from moons_b200 import mesh_gen as mg
from moons_b200 import capi as G
from moons_b200.capi import CC, FX, FY, FZ, EX, EY, EZ, NODE  # noqa: F401

FACES = (FX, FY, FZ)
EDGES = (EX, EY, EZ)


def coords(kind: str, n: int, lo=0.0, hi=1.0, beta=1.05):
    if kind == "uniform":
        h = mg.uniform(lo, hi, n)
    else:
        h = mg.roberts_both(lo, hi, n, beta)
    return mg.add_ghost_nodes(h)


def small_mesh_coords(seed=0, n=(12, 10, 8), stretched=True):
    kinds = ("roberts", "uniform", "roberts") if stretched else ("uniform",) * 3
    return [coords(k, nn, 0.0, 1.0 + 0.5 * i, 1.05 + 0.1 * i) for i, (k, nn) in enumerate(zip(kinds, n))]


def rand(shape, rng):
    return rng.standard_normal(shape)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / den


def bc(types, **kw):
    return G.bc_spec(types, **kw)
