"""The oracle's time schemes of the momentum and induction steps, solve_method
1 to 8 (time_marching_methods.f90:47-208, :266-366), and the RK stage loop of
solve_MOONS (MOONS_solver.f90:73-97), on the CPU.

Properties that pin each scheme's arithmetic without a second implementation:
* the implicit schemes (5, 6, 7) integrate the same equations, so over a fixed
  interval their increments agree to O(dt): the disagreement halves with dt;
* with a zero implicit coefficient the implicit operator is the identity, so
  Euler_time_Euler_sources (5) reduces to Euler_time_no_diff_Euler_sources (3)
  and Euler_time_AB2_sources (6) to Euler_time_no_diff_AB2_sources (4);
* every scheme but the two "no_correction" ones ends divergence-free;
* the "no_correction" schemes (1, 2) are one explicit update: over one step
  the velocity increment is linear in dt, and AB2's first step (Fnm1 = 0) is
  exactly 1.5 times Euler's;
* one inactive RK stage of Euler_time_RK_sources (8, all coefficients 1) is,
  on the first step (Fnm1 = L = 0), Euler_time_Euler_sources with twice the
  implicit coefficient, bit for bit; three stages are consistent with the
  default scheme and end divergence-free;
* the diffusion_linear terms enter through L: on the first step of
  Euler_time_AB2_sources the diffusion through F (AB2: 1.5 F) moves the state
  1.5 times as far as the same diffusion through L;
* Euler_time_AB2_sources_FFT (9) is 6 with a direct cleaning solve, so the
  oracle runs it as 6;
* the energy schemes (solve_energy, energy_extend.f90:244-257): the
  explicit ones (1, 2) are linear in dt with AB2's first step 1.5 times
  Euler's; BDF2 (4) and RK3 (5, all diffusion implicit) agree with the
  implicit AB2 scheme (3) to O(dt);
* a scheme number outside 0..9 (1..5 for the energy), or a stage count
  other than 1 or 3, is refused at create, as the reference's select case
  stops."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import configs
from moons_b200.capi import IND_B, MHD_U, MHD_B, MHD_T

LDC = dict(n=6, induction=IND_B)


def with_params(builder, **fields):
    """builder whose parameters get ``fields`` (callables take the params)."""
    def b(*a, **kw):
        mom, ind, prm, init = builder(*a, **kw)
        for k, v in fields.items():
            setattr(prm, k, v(prm) if callable(v) else v)
        return mom, ind, prm, init
    return b


# explicit diffusion (beta = 1, var_set_extend.f90:55-86): F_U += (1/Re) lap U,
# F_B += -curl(sigma^-1 J)
explicit_diffusion = dict(scale_diffusion_U=lambda p: -p.coeff_implicit_U, scale_diffusion_B=-1.0)


def run(method, dt, nsteps, builder=configs.ldc, **kw):
    sim = configs.make(O, builder, seed=3, dt=dt, tol=1e-12, solve_method_U=method, solve_method_B=method,
                       **(kw or LDC))
    u0 = [sim.download(MHD_U, c).copy() for c in range(3)]
    b0 = [sim.download(MHD_B, c).copy() for c in range(3)]
    sim.step(nsteps)
    du = np.concatenate([(sim.download(MHD_U, c) - u0[c]).ravel() for c in range(3)])
    db = np.concatenate([(sim.download(MHD_B, c) - b0[c]).ravel() for c in range(3)])
    return sim, du, db


@pytest.mark.parametrize("field", ["solve_method_U", "solve_method_B"])
@pytest.mark.parametrize("bad", [-1, 10])
def test_unknown_scheme_refused(field, bad):
    mom, ind, prm, _ = configs.ldc(n=6, induction=IND_B)
    setattr(prm, field, bad)
    mm = O.Mesh(*mom)
    with pytest.raises(ValueError):
        O.MHD(mm, mm, prm)


def test_implicit_schemes_agree_to_first_order_in_dt():
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


@pytest.mark.parametrize("explicit,implicit", [(3, 5), (4, 6)])
def test_implicit_scheme_reduces_to_explicit_at_zero_coefficient(explicit, implicit):
    b = with_params(configs.ldc, coeff_implicit_U=0.0, coeff_implicit_B=0.0)
    se, due, dbe = run(explicit, 1e-3, 4, b, **LDC)
    si, dui, dbi = run(implicit, 1e-3, 4, b, **LDC)
    assert np.linalg.norm(due - dui) <= 1e-8 * np.linalg.norm(dui)
    assert np.linalg.norm(dbe - dbi) <= 1e-8 * np.linalg.norm(dbi)
    duv, dbv = se.divergence()
    assert duv < 1e-18 and dbv < 1e-18


def test_no_correction_schemes_are_one_explicit_update():
    b = with_params(configs.ldc, **explicit_diffusion)
    _, du1, _ = run(1, 1e-3, 1, b, **LDC)
    _, du1b, _ = run(1, 2e-3, 1, b, **LDC)
    _, du2, _ = run(2, 1e-3, 1, b, **LDC)
    _, du2b, _ = run(2, 2e-3, 1, b, **LDC)
    assert np.linalg.norm(du1) > 0
    assert np.linalg.norm(du1b - 2 * du1) <= 1e-11 * np.linalg.norm(du1b)
    assert np.linalg.norm(du2b - 2 * du2) <= 1e-11 * np.linalg.norm(du2b)
    # AB2(F, Fnm1) = 1.5 F - 0.5 Fnm1 with Fnm1 = 0 on the first step
    assert np.linalg.norm(du2 - 1.5 * du1) <= 1e-11 * np.linalg.norm(du2)


@pytest.mark.parametrize("stages", [2, 4])
def test_unknown_stage_count_refused(stages):
    mom, ind, prm, _ = configs.ldc(n=6, induction=IND_B)
    prm.rk_stages = stages
    mm = O.Mesh(*mom)
    with pytest.raises(ValueError):
        O.MHD(mm, mm, prm)


@pytest.mark.parametrize("bad", [0, 6])
def test_unknown_energy_scheme_refused(bad):
    mom, ind, prm, _ = configs.ldc_energy(n=6, solve_method_T=bad)
    mm = O.Mesh(*mom)
    with pytest.raises(ValueError):
        O.MHD(mm, mm, prm)


def test_inactive_rk_stage_is_euler_with_twice_the_coefficient():
    b8 = with_params(configs.ldc, rk_stages=1)
    b5 = with_params(configs.ldc, coeff_implicit_U=lambda p: 2 * p.coeff_implicit_U,
                     coeff_implicit_B=lambda p: 2 * p.coeff_implicit_B)
    _, du8, db8 = run(8, 1e-3, 1, b8, **LDC)
    _, du5, db5 = run(5, 1e-3, 1, b5, **LDC)
    assert np.linalg.norm(du5) > 0 and np.linalg.norm(db5) > 0
    assert np.array_equal(du8, du5) and np.array_equal(db8, db5)


def test_rk3_is_consistent_with_the_default_scheme():
    T = 8e-3
    gaps = []
    for dt in (2e-3, 1e-3):
        n = int(round(T / dt))
        _, d6, _ = run(6, dt, n)
        sim, d8, _ = run(8, dt, n, with_params(configs.ldc, rk_stages=3), **LDC)
        duv, dbv = sim.divergence()
        assert duv < 1e-18 and dbv < 1e-18
        gaps.append(np.linalg.norm(d8 - d6) / np.linalg.norm(d6))
    assert gaps[0] < 0.05 and gaps[1] < 0.75 * gaps[0], gaps


def test_linear_diffusion_enters_through_L():
    s_u = lambda p: -p.coeff_implicit_U  # noqa: E731
    _, d0, b0 = run(6, 1e-3, 1)
    _, dF, bF = run(6, 1e-3, 1, with_params(configs.ldc, scale_diffusion_U=s_u, scale_diffusion_B=-1.0), **LDC)
    _, dL, bL = run(6, 1e-3, 1, with_params(configs.ldc, scale_diffusion_linear_U=s_u,
                                            scale_diffusion_linear_B=-1.0), **LDC)
    assert np.linalg.norm(dF - d0) > 0 and np.linalg.norm(bF - b0) > 0
    assert np.linalg.norm((dF - d0) - 1.5 * (dL - d0)) <= 1e-10 * np.linalg.norm(dF - d0)
    assert np.linalg.norm((bF - b0) - 1.5 * (bL - b0)) <= 1e-9 * np.linalg.norm(bF - b0)


def test_fft_scheme_runs_the_default_arithmetic():
    _, du6, db6 = run(6, 1e-3, 2)
    _, du9, db9 = run(9, 1e-3, 2)
    assert np.array_equal(du6, du9) and np.array_equal(db6, db9)


def run_T(mT, dt, nsteps, rk=0, implicit_only=False):
    """heated cavity (6^3): the temperature increment after nsteps."""
    def b(*a, **kw):
        mom, ind, prm, init = configs.ldc_energy(*a, **kw)
        prm.rk_stages = rk
        if implicit_only:  # all diffusion in the solve: beta sums to 1/2 over the stages
            prm.scale_diffusion_T = 0.0
            prm.coeff_implicit_T = 2 * prm.coeff_implicit_T
        return mom, ind, prm, init
    sim = configs.make(O, b, seed=3, n=6, dt=dt, tol=1e-12, solve_method_T=mT, solve_method_U=8 if rk == 3 else 0)
    t0 = sim.download(MHD_T, 0).copy()
    sim.step(nsteps)
    return (sim.download(MHD_T, 0) - t0).ravel()


def test_explicit_energy_schemes_are_one_explicit_update():
    d1, d1b, d2 = run_T(1, 1e-3, 1), run_T(1, 2e-3, 1), run_T(2, 1e-3, 1)
    assert np.linalg.norm(d1) > 0
    assert np.linalg.norm(d1b - 2 * d1) <= 1e-11 * np.linalg.norm(d1b)
    assert np.linalg.norm(d2 - 1.5 * d1) <= 1e-11 * np.linalg.norm(d2)


def test_implicit_energy_schemes_agree_to_first_order_in_dt():
    T = 8e-3
    gaps = {4: [], 5: []}
    for dt in (2e-3, 1e-3):
        n = int(round(T / dt))
        d3 = run_T(3, dt, n)
        gaps[4].append(np.linalg.norm(run_T(4, dt, n) - d3) / np.linalg.norm(d3))
        gaps[5].append(np.linalg.norm(run_T(5, dt, n, rk=3, implicit_only=True) - d3) / np.linalg.norm(d3))
    for m, g in gaps.items():
        assert g[0] < 0.2 and g[1] < 0.75 * g[0], (m, g)
