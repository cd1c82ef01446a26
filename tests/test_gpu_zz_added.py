"""GPU tests added after the other GPU test files had last run on a B200:
the energy schemes 1, 4 and 5 of solve_energy, Euler_time_AB2_sources_FFT
(solve_method 9: the default scheme with the cleaning equations solved
directly), the refusal of Poisson solver choices the step cannot use, and
Hunt's duct profile.  Collected after the other GPU test files so that a
failure here cannot stop the rest of the suite under -x; the arithmetic of
every RHS form is also checked on the CPU (tests/test_emu_cpu.py), the
oracle's schemes by property tests (tests/test_time_schemes_cpu.py) and its
Hunt profile by tests/test_known_answer_cpu.py."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200 import configs
from tests import known_answers as KA

pytestmark = pytest.mark.gpu

# the step test's LDC in the B form and duct with walls (tests/test_gpu_mhd.py)
SCHEME_CASES = [
    ("ldc_bform", configs.ldc, dict(n=10, induction=G.IND_B, tol=1e-12)),
    ("duct_walls", configs.duct, dict(nx=10, ny=8, nz=12, n_wall=2, t_wall=0.5, tol=1e-12, noise=1e-2)),
]


def rel_l2(a, b):
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


@pytest.mark.parametrize("mT", [1, 4, 5])
def test_mhd_energy_time_schemes_match_oracle(mT):
    """The energy schemes 1, 4 and 5 of solve_energy (energy_extend.f90:
    244-257, time_marching_methods_SF.f90): 4 steps of the heated cavity
    against the oracle running the same scheme, every field within 1e-10.
    Scheme 5 runs three RK stages (momentum with Euler_time_RK_sources) and
    takes half its diffusion explicitly through L."""
    def builder(*a, **kw):
        mom, ind, prm, init = configs.ldc_energy(*a, **kw)
        prm.rk_stages = 3 if mT == 5 else 0
        return mom, ind, prm, init
    kw = dict(n=10, tol=1e-12, solve_method_T=mT, solve_method_U=8 if mT == 5 else 0)
    g = configs.make(G, builder, seed=3, **kw)
    o = configs.make(O, builder, seed=3, **kw)
    nsteps = 4
    ig = g.step(nsteps)
    io = o.step(nsteps)
    fields = ([(G.MHD_U, c) for c in range(3)] + [(G.MHD_P, 0), (G.MHD_T, 0), (G.MHD_PHI, 0)] +
              [(G.MHD_J, c) for c in range(3)] + [(G.MHD_JXB, c) for c in range(3)])
    for which, c in fields:
        e = rel_l2(g.download(which, c), o.download(which, c))
        assert e < 1e-10, f"energy scheme {mT}: field {which}/{c} rel L2 {e}"
    nsolves = nsteps * (3 if mT == 5 else 1)
    for k in ("iters_U", "iters_p", "iters_phi", "iters_T"):
        assert abs(ig[k] - io[k]) <= max(nsolves, 0.005 * io[k]), (k, ig, io)


@pytest.mark.parametrize("name,builder,kw", SCHEME_CASES, ids=[c[0] for c in SCHEME_CASES])
def test_mhd_fft_scheme_direct_cleaning(name, builder, kw):
    """solve_method 9 (Euler_time_AB2_sources_FFT, time_marching_methods.f90:
    152-185): the default scheme with the cleaning equations solved directly
    (clean_div_FFT), here by the fast-diagonalization solve.  Against the
    oracle's Jacobi-PCG cleaning, both to 1e-12: fields agree to solver
    accuracy (the bound of the direct-solve step test) and each cleaning
    solve takes a few CG iterations at most."""
    g = configs.make(G, builder, seed=3, solve_method_U=9, solve_method_B=9, **kw)
    o = configs.make(O, builder, seed=3, **kw)
    nsteps = 4
    ig = g.step(nsteps)
    o.step(nsteps)
    fields = ([(G.MHD_U, c) for c in range(3)] + [(G.MHD_B, c) for c in range(3)] +
              [(G.MHD_J, c) for c in range(3)] + [(G.MHD_JXB, c) for c in range(3)])
    for which, c in fields:
        e = rel_l2(g.download(which, c), o.download(which, c))
        assert e < 1e-7, f"{name}: field {which}/{c} rel L2 {e}"
    dug, dbg = g.divergence()
    duo, dbo = o.divergence()
    assert dug <= max(100 * duo, 1e-22)
    assert dbg <= max(100 * dbo, 1e-22)
    # at most three CG iterations per direct-preconditioned solve, the bound of
    # the direct solve's own test (hundreds with the Jacobi preconditioner)
    assert ig["iters_p"] <= 3 * nsteps and ig["iters_phi"] <= 3 * nsteps, ig


@pytest.mark.parametrize("bad", [G.PREC_MOM, G.PREC_UNET, 9])
def test_mhd_rejects_unknown_poisson_solver(bad):
    """prec_poisson values the step cannot use are refused, not replaced."""
    mom, ind, prm, _ = configs.ldc(n=6)
    prm.prec_poisson = bad
    mm = G.Mesh(*mom)
    with pytest.raises(G.MoonsError) as e:
        G.MHD(mm, mm, prm)
    assert e.value.code == 1  # MOONS_ERR_ARG


def test_hunt_profile_second_order_gpu():
    """The steady duct with conducting Hartmann walls reproduces Hunt's
    profile (profile_funcs.f90:147-193) at second order (oracle: 0.0465,
    0.0110, 0.0027 at 8, 16, 32 cells)."""
    errs = [KA.duct_steady(G, n, walls="hunt")[0] for n in (16, 32, 64)]
    assert errs[-1] < 1.5e-3, errs
    for a, b in zip(errs, errs[1:]):
        assert a / b > 3.5, errs
