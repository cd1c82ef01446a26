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


def test_sigma_laplacian_series_resistance():
    """div(k grad phi) = 0 (Lap_nonuniform_props, matrix_free_operators.f90:
    92-118) with phi = 1 on x = 0, phi = 0 on x = 1, insulated elsewhere and k
    varying along x on the x-faces: the discrete solution is resistances in
    series, R_f = dx / k_f, the Dirichlet walls entering through half their
    face's resistance (ghost 2 b - phi_1).  Solved by the oracle's Jacobi-PCG."""
    from moons_b200 import mesh_gen as mg
    from moons_b200.capi import CC, DIRICHLET, FX, FY, FZ, NEUMANN, OP_LAP_PROPS, PREC_LAP, bc_spec, isp
    n = 8
    h = mg.add_ghost_nodes(mg.uniform(0.0, 1.0, n))
    m = O.Mesh(h, h.copy(), h.copy())
    phi = m.field(CC)
    phi.upload(np.zeros(phi.shape))
    phi.set_bcs(bc_spec([DIRICHLET, DIRICHLET, NEUMANN, NEUMANN, NEUMANN, NEUMANN], values=[1.0, 0, 0, 0, 0, 0]))
    kx = 1.0 + 0.5 * np.sin(3.0 * h)
    ks = []
    for dl in (FX, FY, FZ):
        f = m.field(dl)
        k = np.ones(f.shape)
        if dl == FX:
            k[:] = kx[:, None, None]
        f.upload(k)
        ks.append(f)
    b = m.field(CC)
    b.upload(np.zeros(b.shape))
    info = O.PCG(m, OP_LAP_PROPS, PREC_LAP, [phi], [phi], ks).solve([phi], [b], isp(2000, 1e-14, 1e-300))
    assert info["exit_reason"] == 1
    R = (h[2] - h[1]) / kx[1:n + 2]
    q = 1.0 / (R[0] / 2 + R[1:-1].sum() + R[-1] / 2)
    expect = 1.0 - q * (R[0] / 2 + np.concatenate([[0.0], np.cumsum(R[1:n])]))
    assert np.abs(phi.download()[1:-1, 1:-1, 1:-1] - expect[:, None, None]).max() <= 1e-12
