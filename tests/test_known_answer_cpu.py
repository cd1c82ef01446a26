"""Known-answer pins of the oracle (CPU): the reference's own verification
routines and analytic solutions, and the configuration-1 golden fixture.

* grad(lap phi) = lap(grad phi) away from the boundary
  (operator_commute_test.f90:52-93) on uniform and Roberts-stretched meshes;
* the steady state of the MHD duct step converges to the Shercliff profile
  (profile_funcs.f90:65-156) at second order in the mesh spacing;
* the Taylor-Green vortex (GF_distributions.f90:720-769) decays at the
  analytic rate, the error first order in dt (backward-Euler diffusion with
  a pressure projection);
* the first 20 steps of configuration 1 (lid-driven cavity 32^3) reproduce
  the fixture ``tests/golden/ldc32_step20.json`` bit for bit, which ties the
  1000-step fixture the GPU tests compare against to this oracle.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from tests import known_answers as KA

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("kind", ["uniform", "roberts"])
def test_grad_lap_commute(kind):
    for n in (8, 16):
        assert KA.grad_lap_commute(O, O, kind, n) < 1e-14


def test_shercliff_profile_second_order():
    e8, _ = KA.duct_steady(O, 8)
    e16, _ = KA.duct_steady(O, 16)
    assert e16 < 0.02, (e8, e16)
    assert e8 / e16 > 3.5, (e8, e16)


def test_hunt_profile_second_order():
    """Conducting Hartmann walls, insulating side walls: Hunt's profile."""
    e8, _ = KA.duct_steady(O, 8, walls="hunt")
    e16, _ = KA.duct_steady(O, 16, walls="hunt")
    assert e16 < 0.02, (e8, e16)
    assert e8 / e16 > 3.5, (e8, e16)


def test_taylor_green_decay_first_order_in_time():
    e1 = KA.taylor_green(O, 16, 2e-3)
    e2 = KA.taylor_green(O, 16, 1e-3)
    assert e1 < 6e-4 and e2 < 3.5e-4, (e1, e2)
    assert 1.6 < e1 / e2 < 2.4, (e1, e2)


def test_ldc32_fixture_is_the_oracle():
    from tests.golden import make_ldc32 as mk
    with open(os.path.join(GOLDEN, "ldc32_step20.json")) as f:
        ref = json.load(f)
    sim = mk.build_case(O)
    info = sim.step(ref["steps"])
    for k, v in ref["iters"].items():
        assert info[k] == v, (k, info[k], v)
    got = mk.digest(sim)
    for name, d in ref["fields"].items():
        assert got[name]["sha256"] == d["sha256"], (name, got[name]["l2"], d["l2"])
    z = np.load(os.path.join(GOLDEN, "ldc32_step1000.npz"))
    assert int(z["steps"]) == 1000
    shapes = {name: sim.shape(which, c) for name, which, c in mk.FIELDS_LONG}
    for name, shp in shapes.items():
        assert z[name].shape == shp
