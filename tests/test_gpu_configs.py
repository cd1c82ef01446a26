"""The stated configurations at their stated sizes, and the known answers,
on the GPU.

* Configuration 1: the MHD lid-driven cavity, uniform 32^3, Re = 400,
  Ha = 10, low-Rem potential form, dt = 1e-3, PCG to 1e-10 relative
  residual, 1000 steps from the seeded state; every field against the
  oracle's 1000-step fixture (``tests/golden/ldc32_step1000.npz``, made by
  ``tests/golden/make_ldc32.py`` and pinned to the oracle by a CPU test)
  within relative L2 1e-10, div U / div B at the oracle's level.
* Configuration 2: the MHD duct at its full size (64 x 64 x 256 fluid
  cells, 4-cell sigma = 0.01 wall layer, Roberts beta = 1.05, Ha = 100,
  Re = 1000, dt = 5e-4, PCG to 1e-10): two steps against the oracle run
  alongside, relative L2 <= 1e-10 per field.
* Known answers: the steady duct step converges to the Shercliff profile at
  second order; the Taylor-Green vortex decays within the oracle's error;
  grad(lap) = lap(grad) to round-off.
"""
import os

import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200 import configs
from tests import known_answers as KA

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-10


def rel_l2(a, b):
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def test_config1_ldc32_1000_steps_match_oracle_fixture():
    from tests.golden import make_ldc32 as mk
    z = np.load(os.path.join(GOLDEN, "ldc32_step1000.npz"))
    sim = mk.build_case(G)
    tot = {"iters_U": 0, "iters_p": 0, "iters_phi": 0}
    for _ in range(10):
        info = sim.step(100)
        for k in tot:
            tot[k] += info[k]
    worst = {}
    for name, which, c in mk.FIELDS_LONG:
        e = rel_l2(sim.download(which, c), z[name])
        worst[name] = e
    assert max(worst.values()) <= TOL, worst
    du, db = sim.divergence()
    assert du <= max(10.0 * float(z["div_u"]), 1e-24), (du, float(z["div_u"]))
    assert db <= max(10.0 * float(z["div_b"]), 1e-24), (db, float(z["div_b"]))
    for k in tot:
        assert abs(tot[k] - int(z[k])) <= 0.01 * int(z[k]) + 10, (k, tot[k], int(z[k]))


def test_config2_duct_full_size_two_steps_match_oracle():
    g = configs.make(G, configs.duct, seed=0)
    o = configs.make(O, configs.duct, seed=0)
    ig = g.step(2)
    io = o.step(2)
    fields = [(G.MHD_U, c) for c in range(3)] + [(G.MHD_P, 0)] + [(G.MHD_B, c) for c in range(3)] + \
             [(G.MHD_J, c) for c in range(3)] + [(G.MHD_JXB, c) for c in range(3)]
    worst = {}
    for which, c in fields:
        worst[(which, c)] = rel_l2(g.download(which, c), o.download(which, c))
    assert max(worst.values()) <= TOL, worst
    dug, dbg = g.divergence()
    duo, dbo = o.divergence()
    assert dug <= max(10 * duo, 1e-24) and dbg <= max(10 * dbo, 1e-24), (dug, duo, dbg, dbo)
    for k in ("iters_U", "iters_p", "iters_B", "iters_phi"):
        assert abs(ig[k] - io[k]) <= 2 + 0.01 * io[k], (k, ig, io)


def test_shercliff_profile_second_order_gpu():
    errs = [KA.duct_steady(G, n)[0] for n in (16, 32, 64)]
    assert errs[-1] < 1.5e-3, errs
    for a, b in zip(errs, errs[1:]):
        assert a / b > 3.5, errs


def test_taylor_green_decay_gpu():
    for dt in (2e-3, 1e-3):
        eg = KA.taylor_green(G, 16, dt)
        eo = KA.taylor_green(O, 16, dt)
        assert abs(eg - eo) <= 1e-6 * eo, (dt, eg, eo)


@pytest.mark.parametrize("kind", ["uniform", "roberts"])
def test_grad_lap_commute_gpu(kind):
    for n in (8, 32):
        assert KA.grad_lap_commute(G, G, kind, n) < 1e-14
