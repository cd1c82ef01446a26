"""Known answers for the oracle's energy equation.

Sources (energy_sources.f90:51-94), through one explicit-Euler energy step
(solve_method_T 1: T += dt F_T) of the heated cavity in the B form on a
uniform 8^3 mesh, with advection, diffusion and heating off so that F_T is
the source under test.  With the shear U_x = a y (faces), the cell-centre
velocity is a y_c, so
  viscous dissipation  sum_cd (d_d U_c)^2      = a^2,
  KE diffusion         lap(sum_c U_c^2) = lap(a^2 y^2) = 2 a^2;
with B_x = b y, J = curl(B) / Rem = (0, 0, -b) (Rem = 1), so
  Joule heating        |J_CC|^2 sigmaInv_CC    = b^2 sigmaInv_CC.
The stencils are exact for these polynomials on a uniform mesh; cells whose
stencils reach the boundary values set by the BCs are left out.

Conduction (nrg_diffusion, matrix_free_operators.f90:148-174, implicit
Euler_time_AB2_sources_SF with steps long enough to reach the steady state):
T = 1 on x = 0, T = 0 on x = 1, insulated elsewhere, no flow terms.  With
k = 1 the steady state is T = 1 - x (exact on the mesh).  With k varying
along x on the x-faces the discrete steady state is resistances in series:
each face carries R_f = dx / k_f, the Dirichlet walls enter through half
their face's resistance (the ghost value 2 b - T_1), and
T_i = 1 - q (R_wall / 2 + sum of the faces between the wall and cell i).
"""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import configs
from moons_b200.capi import IND_B, MHD_B, MHD_KT, MHD_SIGMA_INV_CC, MHD_T, MHD_U

A, B, DT = 0.7, 0.9, 1e-3


def source_rate(ke=0.0, visc=0.0, joule=0.0, sig=1.0):
    def builder(*args, **kw):
        mom, ind, prm, init = configs.ldc_energy(*args, **kw)
        prm.scale_advection_T = 0.0
        prm.scale_diffusion_T = 0.0
        prm.scale_heating_T = 0.0

        def init2(sim, rng):
            init(sim, rng)
            h = mom[1]
            yc = 0.5 * (h[1:] + h[:-1])
            for c in range(3):
                u = np.zeros(sim.shape(MHD_U, c))
                bb = np.zeros(sim.shape(MHD_B, c))
                if c == 0:
                    u[:] = A * yc[None, :, None]
                    bb[:] = B * yc[None, :, None]
                sim.upload(MHD_U, c, u)
                sim.upload(MHD_B, c, bb)
            sim.upload(MHD_SIGMA_INV_CC, 0, np.full(sim.shape(MHD_SIGMA_INV_CC), sig))
        return mom, ind, prm, init2

    sim = configs.make(O, builder, seed=3, n=8, dt=DT, tol=1e-12, induction=IND_B, solve_method_T=1,
                       KE_diffusion=ke, viscous_dissipation=visc, joule_heating=joule)
    t0 = sim.download(MHD_T, 0).copy()
    sim.step(1)
    return ((sim.download(MHD_T, 0) - t0) / DT)[3:-3, 3:-3, 3:-3]


@pytest.mark.parametrize("kw,expect", [(dict(visc=1.0), A * A), (dict(ke=1.0), 2 * A * A),
                                       (dict(joule=1.0, sig=1.3), B * B * 1.3), (dict(visc=0.5, ke=2.0), 4.5 * A * A)])
def test_energy_source_known_answer(kw, expect):
    r = source_rate(**kw)
    assert r.size > 0
    assert np.abs(r - expect).max() <= 1e-10 * expect, (r.min(), r.max(), expect)


def steady_conduction(kx_nodes=None, n=8):
    def builder(*args, **kw):
        mom, ind, prm, init = configs.ldc_energy(*args, **kw)
        prm.scale_advection_T = 0.0
        prm.scale_heating_T = 0.0
        prm.scale_advection_U = 0.0   # keeps the momentum step bounded at these steps
        prm.scale_buoyancy = 0.0

        def init2(sim, rng):
            init(sim, rng)
            for c in range(3):
                k = np.ones(sim.shape(MHD_KT, c))
                if c == 0 and kx_nodes is not None:
                    k[:] = kx_nodes[:, None, None]
                sim.upload(MHD_KT, c, k)
        return mom, ind, prm, init2

    sim = configs.make(O, builder, seed=3, n=n, dt=1e6, tol=1e-13, solve_method_T=3)
    sim.step(3)
    return sim.download(MHD_T, 0)


def test_steady_conduction_is_linear():
    n = 8
    h = configs.ldc(n=n)[0][0]
    xc = 0.5 * (h[1:] + h[:-1])
    T = steady_conduction(n=n)
    assert np.abs(T[1:-1, 1:-1, 1:-1] - (1.0 - xc)[1:-1, None, None]).max() <= 1e-12


def test_steady_conduction_resistances_in_series():
    n = 8
    h = configs.ldc(n=n)[0][0]      # x nodes with ghosts: the walls are h[1] and h[n + 1]
    kx = 1.0 + 0.5 * np.sin(3.0 * h)
    T = steady_conduction(kx, n=n)
    R = (h[2] - h[1]) / kx[1:n + 2]
    q = 1.0 / (R[0] / 2 + R[1:-1].sum() + R[-1] / 2)
    expect = 1.0 - q * (R[0] / 2 + np.concatenate([[0.0], np.cumsum(R[1:n])]))
    assert np.abs(T[1:-1, 1:-1, 1:-1] - expect[:, None, None]).max() <= 1e-12
