"""Known answers for the oracle's energy sources (energy_sources.f90:51-94),
through one explicit-Euler energy step (solve_method_T 1: T += dt F_T) of
the heated cavity in the B form on a uniform 8^3 mesh, with advection,
diffusion and heating off so that F_T is the source under test.

With the shear U_x = a y (faces), the cell-centre velocity is a y_c, so
  viscous dissipation  sum_cd (d_d U_c)^2      = a^2,
  KE diffusion         lap(sum_c U_c^2) = lap(a^2 y^2) = 2 a^2;
with B_x = b y, J = curl(B) / Rem = (0, 0, -b) (Rem = 1), so
  Joule heating        |J_CC|^2 sigmaInv_CC    = b^2 sigmaInv_CC.
The stencils are exact for these polynomials on a uniform mesh; cells whose
stencils reach the boundary values set by the BCs are left out."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import configs
from moons_b200.capi import IND_B, MHD_B, MHD_SIGMA_INV_CC, MHD_T, MHD_U

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
