"""The oracle's three implicit time schemes of the momentum and induction
steps (solve_method 5, 6, 7: Euler_time_Euler_sources, Euler_time_AB2_sources,
O2_BDF_time_AB2_sources, time_marching_methods.f90:47-150), on the CPU.

Properties that hold whatever the scheme: each step ends divergence-free
(clean_div with its scale), and the three schemes integrate the same
equations, so over a fixed interval their increments agree to O(dt) and the
disagreement shrinks as dt does.  A scheme number outside 0, 5, 6, 7 is
refused at create, as the reference's select case stops."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import configs
from moons_b200.capi import IND_B, MHD_U, MHD_B


def run(method, dt, nsteps):
    sim = configs.make(O, configs.ldc, seed=3, n=6, induction=IND_B, dt=dt, tol=1e-12,
                       solve_method_U=method, solve_method_B=method)
    u0 = [sim.download(MHD_U, c).copy() for c in range(3)]
    b0 = [sim.download(MHD_B, c).copy() for c in range(3)]
    sim.step(nsteps)
    du = np.concatenate([(sim.download(MHD_U, c) - u0[c]).ravel() for c in range(3)])
    db = np.concatenate([(sim.download(MHD_B, c) - b0[c]).ravel() for c in range(3)])
    return sim, du, db


@pytest.mark.parametrize("field", ["solve_method_U", "solve_method_B"])
def test_unknown_scheme_refused(field):
    mom, ind, prm, _ = configs.ldc(n=6, induction=IND_B)
    setattr(prm, field, 8)
    mm = O.Mesh(*mom)
    with pytest.raises(ValueError):
        O.MHD(mm, mm, prm)


def test_schemes_agree_to_first_order_in_dt():
    T = 8e-3
    gaps = []
    for dt in (2e-3, 1e-3):
        n = int(round(T / dt))
        runs = {m: run(m, dt, n) for m in (5, 6, 7)}
        for m, (sim, du, db) in runs.items():
            duv, dbv = sim.divergence()
            assert duv < 1e-18 and dbv < 1e-18, (m, dt, duv, dbv)
            assert np.linalg.norm(du) > 0
        ref_u = np.linalg.norm(runs[6][1])
        gap = max(np.linalg.norm(runs[m][1] - runs[6][1]) / ref_u for m in (5, 7))
        gaps.append(gap)
        assert gap < 0.2, (dt, gap)
    # halving dt halves (about) the disagreement between the schemes
    assert gaps[1] < 0.75 * gaps[0], gaps
