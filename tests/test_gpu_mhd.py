"""GPU parity of the full MHD time step against the oracle.

Small versions of the benchmark cases (same presets, coarser meshes) run
N steps on both sides from the same seeded state.  Solver tolerances are
tightened to 1e-12 so the comparison measures the kernels, not the stopping
point: per-field relative L2 <= 1e-10 after the steps, and div U, div B at
the oracle's level."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200 import configs

pytestmark = pytest.mark.gpu

CASES = [
    ("ldc_potential", configs.ldc, dict(n=10, induction=G.IND_POTENTIAL, tol=1e-12)),
    ("ldc_bform", configs.ldc, dict(n=10, induction=G.IND_B, tol=1e-12)),
    ("duct_walls", configs.duct, dict(nx=10, ny=8, nz=12, n_wall=2, t_wall=0.5, tol=1e-12, noise=1e-2)),
    ("duct_nowall", configs.duct, dict(nx=8, ny=8, nz=12, n_wall=0, tol=1e-12, noise=1e-2)),
    # configuration 5's physics (Ha = 500, Rem = 10, dt = 2e-4) on a small grid
    ("at_scale_small", configs.at_scale, dict(nx=8, ny=8, nz=16, tol=1e-12)),
    # the energy equation (implicit and explicit diffusion), buoyancy into momentum
    ("ldc_energy_implicit", configs.ldc_energy, dict(n=10, tol=1e-12, solve_method_T=3)),
    ("ldc_energy_explicit", configs.ldc_energy, dict(n=10, tol=1e-12, solve_method_T=2)),
    # the KE-diffusion, viscous-dissipation and Joule-heating sources
    # (energy_sources.f90:51-94), B form (J on edges) and potential form
    ("ldc_energy_sources_bform", configs.ldc_energy, dict(n=10, tol=1e-12, induction=G.IND_B, KE_diffusion=0.3,
                                                          viscous_dissipation=0.2, joule_heating=0.4)),
    ("ldc_energy_sources_potential", configs.ldc_energy, dict(n=10, tol=1e-12, KE_diffusion=0.3,
                                                              viscous_dissipation=0.2, joule_heating=0.4)),
    # the full_BC case on mesh-bank meshes: clustered fluid embedded in an
    # induction mesh with thin walls and a vacuum region (sigma = 1e-3)
    ("full_bc_vacuum", configs.full_bc, dict(N=8, N_w=3, tol=1e-12, iter_max=(20000,) * 4, noise=1e-2)),
]


def rel_l2(a, b):
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


@pytest.mark.parametrize("name,builder,kw", CASES, ids=[c[0] for c in CASES])
def test_mhd_steps_match_oracle(name, builder, kw):
    g = configs.make(G, builder, seed=3, **kw)
    o = configs.make(O, builder, seed=3, **kw)
    nsteps = 4
    ig = g.step(nsteps)
    io = o.step(nsteps)
    fields = [(G.MHD_U, c) for c in range(3)] + [(G.MHD_P, 0), (G.MHD_JXB, 0), (G.MHD_JXB, 1), (G.MHD_JXB, 2)]
    ind = kw.get("induction", G.IND_POTENTIAL if builder in (configs.ldc, configs.ldc_energy) else G.IND_B)
    if builder is configs.ldc_energy:
        fields += [(G.MHD_T, 0)]
    if ind != G.IND_OFF:
        fields += [(G.MHD_J, c) for c in range(3)]
    if ind == G.IND_POTENTIAL:
        fields += [(G.MHD_PHI, 0)]
    if ind == G.IND_B:
        # the cleaning potential of the B form is a Lagrange multiplier at
        # round-off level (div B* ~ 1e-17), so it is not compared
        fields += [(G.MHD_B, c) for c in range(3)]
    for which, c in fields:
        a, b = g.download(which, c), o.download(which, c)
        e = rel_l2(a, b)
        assert e < 1e-10, f"{name}: field {which}/{c} rel L2 {e}"
    dug, dbg = g.divergence()
    duo, dbo = o.divergence()
    assert dug <= max(10 * duo, 1e-24)
    assert dbg <= max(10 * dbo, 1e-24)
    # iteration counts: within one per solve, or 0.5% for solves of
    # hundreds of iterations (whose last iteration moves with the order of
    # the floating-point sums)
    for k in ("iters_U", "iters_p", "iters_B", "iters_phi", "iters_T"):
        assert abs(ig[k] - io[k]) <= max(nsteps, 0.005 * io[k]), (k, ig, io)


@pytest.mark.parametrize("prec", [G.PREC_MG, G.PREC_MG_MIXED, G.PREC_FD], ids=["mg", "mixed", "fd"])
@pytest.mark.parametrize("name,builder,kw", [CASES[0], CASES[2], CASES[4]], ids=[CASES[0][0], CASES[2][0], CASES[4][0]])
def test_mhd_steps_multigrid_poisson(name, builder, kw, prec):
    """The step with multigrid-preconditioned pressure/potential solves reaches
    the same fields as the oracle's Jacobi-PCG step: the solves converge to the
    same tolerance, so velocities and currents agree to solver accuracy (the
    pressure itself may differ by a constant in all-Neumann problems)."""
    mom, ind, prm, init = builder(**kw)
    prm.prec_poisson = prec
    mm = G.Mesh(*mom)
    mi = mm if ind is mom else G.Mesh(*ind)
    g = G.MHD(mm, mi, prm)
    init(g, np.random.default_rng(3))
    g.init()
    o = configs.make(O, builder, seed=3, **kw)
    nsteps = 4
    ig = g.step(nsteps)
    o.step(nsteps)
    fields = [(G.MHD_U, c) for c in range(3)] + [(G.MHD_JXB, c) for c in range(3)] + [(G.MHD_J, c) for c in range(3)]
    for which, c in fields:
        e = rel_l2(g.download(which, c), o.download(which, c))
        assert e < 1e-7, f"{name}: field {which}/{c} rel L2 {e}"
    dug, _ = g.divergence()
    duo, _ = o.divergence()
    assert dug <= max(100 * duo, 1e-22)
    assert ig["iters_p"] < 40 * nsteps


SCHEME_CASES = [CASES[1], CASES[2]]  # LDC in the B form, the duct with walls


def explicit_diffusion(builder):
    """builder with the diffusion terms in the sources (beta = 1,
    var_set_extend.f90:55-86), as the schemes without a diffusion solve use."""
    def b(*a, **kw):
        mom, ind, prm, init = builder(*a, **kw)
        prm.scale_diffusion_U = -prm.coeff_implicit_U
        prm.scale_diffusion_B = -1.0
        return mom, ind, prm, init
    return b


def rk3_linear_diffusion(builder):
    """builder with three RK stages (MOONS_solver.f90:73-97) and the
    diffusion_linear terms, whose L Euler_time_RK_sources weighs by 2 alpha:
    half the diffusion explicit through L, the implicit solve keeps its own."""
    def b(*a, **kw):
        mom, ind, prm, init = builder(*a, **kw)
        prm.rk_stages = 3
        prm.scale_diffusion_linear_U = -0.5 * prm.coeff_implicit_U
        prm.scale_diffusion_linear_B = -0.5
        return mom, ind, prm, init
    return b


@pytest.mark.parametrize("method", [1, 2, 3, 4, 5, 7, 8])
@pytest.mark.parametrize("name,builder,kw", SCHEME_CASES, ids=[c[0] for c in SCHEME_CASES])
def test_mhd_time_schemes_match_oracle(name, builder, kw, method):
    """solve_method 1 to 5, 7 and 8 (time_marching_methods.f90:47-208,
    :266-366) for both the momentum and the induction step: 4 steps against
    the oracle's restatement of the same schemes, every field within the step
    test's 1e-10.  The schemes without a diffusion solve (1 to 4) take the
    diffusion in the sources; Euler_time_RK_sources (8) runs three RK stages
    per step with the diffusion_linear terms in L."""
    if method <= 4:
        builder = explicit_diffusion(builder)
    if method == 8:
        builder = rk3_linear_diffusion(builder)
    g = configs.make(G, builder, seed=3, solve_method_U=method, solve_method_B=method, **kw)
    o = configs.make(O, builder, seed=3, solve_method_U=method, solve_method_B=method, **kw)
    nsteps = 4
    ig = g.step(nsteps)
    io = o.step(nsteps)
    fields = ([(G.MHD_U, c) for c in range(3)] + [(G.MHD_P, 0)] + [(G.MHD_B, c) for c in range(3)] +
              [(G.MHD_J, c) for c in range(3)] + [(G.MHD_JXB, c) for c in range(3)])
    for which, c in fields:
        e = rel_l2(g.download(which, c), o.download(which, c))
        assert e < 1e-10, f"{name} method {method}: field {which}/{c} rel L2 {e}"
    dug, dbg = g.divergence()
    duo, dbo = o.divergence()
    assert dug <= max(10 * duo, 1e-24)
    assert dbg <= max(10 * dbo, 1e-24)
    nsolves = nsteps * (3 if method == 8 else 1)  # one solve per RK stage
    for k in ("iters_U", "iters_p", "iters_B", "iters_phi"):
        assert abs(ig[k] - io[k]) <= max(nsolves, 0.005 * io[k]), (k, ig, io)


@pytest.mark.parametrize("field", ["solve_method_U", "solve_method_B"])
def test_mhd_rejects_unknown_time_scheme(field):
    mom, ind, prm, _ = configs.ldc(n=6, induction=G.IND_B)
    setattr(prm, field, 10)
    mm = G.Mesh(*mom)
    with pytest.raises(G.MoonsError) as e:
        G.MHD(mm, mm, prm)
    assert e.value.code == 1  # MOONS_ERR_ARG


@pytest.mark.parametrize("stages", [2, 4])
def test_mhd_rejects_bad_rk_stages(stages):
    mom, ind, prm, _ = configs.ldc(n=6, induction=G.IND_B)
    prm.rk_stages = stages
    mm = G.Mesh(*mom)
    with pytest.raises(G.MoonsError) as e:
        G.MHD(mm, mm, prm)
    assert e.value.code == 1  # MOONS_ERR_ARG


@pytest.mark.parametrize("bad", [0, 6])
def test_mhd_rejects_unknown_energy_scheme(bad):
    mom, ind, prm, _ = configs.ldc_energy(n=6, solve_method_T=bad)
    mm = G.Mesh(*mom)
    with pytest.raises(G.MoonsError) as e:
        G.MHD(mm, mm, prm)
    assert e.value.code == 1  # MOONS_ERR_ARG
