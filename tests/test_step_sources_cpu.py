"""Known answers for the oracle's momentum and induction sources through one
explicit step (solve_method 1, Euler_time_no_diff_Euler_sources_no_correction:
X += dt F) of the lid-driven cavity on a uniform 8^3 mesh, with the implicit
diffusion off, so that the change of U or B is dt times the source.

* convection (advect_U_convection1, ops_advect.f90:71-127, scale -1): the
  stagnation flow U = (a x, -a y, 0) is divergence-free with
  (u.grad)u = (a^2 x, a^2 y, 0), so dU/dt = -(a^2 x, a^2 y, 0);
* Lorentz force (compute_JCrossB, extract_add_JCrossB, B form): U = 0 and
  B_x = b y give J = curl(B) / Rem = (0, 0, -b) (Rem = 1); with the applied
  B0 = (0, 1, 0) (finite_Rem off, Btot = B0), J x B0 = (b, 0, 0) and
  dU/dt = (N b, 0, 0), N = Ha^2 / Re;
* constrained-transport induction (add_curl_U_cross_B, induction_sources.f90:
  28-38, scale 1): U = (a y, 0, 0), B = 0, B0 = (0, 1, 0) give
  U x B0 = (0, 0, a y) and dB/dt = curl(U x B0) = (a, 0, 0).
The stencils are exact for these polynomials on a uniform mesh; points whose
stencils reach the boundary values set by the BCs are left out."""
import numpy as np

import oracle.oracle as O
from moons_b200 import configs
from moons_b200.capi import IND_B, IND_OFF, MHD_B, MHD_U

A, B, DT, N_CELLS = 0.7, 0.9, 1e-3, 8
RE, HA = 400.0, 10.0


def rate(advect, induction):
    h = configs.ldc(n=N_CELLS)[0][0]
    hc = 0.5 * (h[1:] + h[:-1])

    def builder(*args, **kw):
        mom, ind, prm, init = configs.ldc(*args, **kw)
        prm.coeff_implicit_U = 0.0

        def init2(sim, rng):
            init(sim, rng)
            for c in range(3):
                u = np.zeros(sim.shape(MHD_U, c))
                if advect and c == 0:
                    u[:] = A * h[:, None, None]    # x-faces: x at the nodes
                if advect and c == 1:
                    u[:] = -A * h[None, :, None]   # y-faces: y at the nodes
                sim.upload(MHD_U, c, u)
                if induction == IND_B:
                    bb = np.zeros(sim.shape(MHD_B, c))
                    if c == 0:
                        bb[:] = B * hc[None, :, None]
                    sim.upload(MHD_B, c, bb)
        return mom, ind, prm, init2

    sim = configs.make(O, builder, seed=3, n=N_CELLS, Re=RE, Ha=HA, dt=DT, tol=1e-12, induction=induction,
                       solve_method_U=1, solve_method_B=1)
    u0 = [sim.download(MHD_U, c).copy() for c in range(3)]
    sim.step(1)
    return h, [(sim.download(MHD_U, c) - u0[c]) / DT for c in range(3)]


def test_convection_known_answer():
    h, r = rate(True, IND_OFF)
    i = slice(3, -3)
    ex = -A * A * h[i]
    assert np.abs(r[0][i, i, i] - ex[:, None, None]).max() <= 1e-10
    assert np.abs(r[1][i, i, i] - ex[None, :, None]).max() <= 1e-10
    assert np.abs(r[2][i, i, i]).max() == 0.0


def test_lorentz_force_known_answer():
    _, r = rate(False, IND_B)
    i = slice(3, -3)
    nb = HA * HA / RE * B
    assert np.abs(r[0][i, i, i] - nb).max() <= 1e-10 * nb
    assert np.abs(r[1][i, i, i]).max() == 0.0 and np.abs(r[2][i, i, i]).max() == 0.0


def test_induction_ct_known_answer():
    h = configs.ldc(n=N_CELLS)[0][0]
    hc = 0.5 * (h[1:] + h[:-1])

    def builder(*args, **kw):
        mom, ind, prm, init = configs.ldc(*args, **kw)
        prm.coeff_implicit_U = 0.0
        prm.coeff_implicit_B = 0.0

        def init2(sim, rng):
            init(sim, rng)
            for c in range(3):
                u = np.zeros(sim.shape(MHD_U, c))
                if c == 0:
                    u[:] = A * hc[None, :, None]   # x-faces: y at the cell centres
                sim.upload(MHD_U, c, u)
                sim.upload(MHD_B, c, np.zeros(sim.shape(MHD_B, c)))
        return mom, ind, prm, init2

    sim = configs.make(O, builder, seed=3, n=N_CELLS, dt=DT, tol=1e-12, induction=IND_B, solve_method_U=1,
                       solve_method_B=1)
    b0 = [sim.download(MHD_B, c).copy() for c in range(3)]
    sim.step(1)
    i = slice(3, -3)
    r = [((sim.download(MHD_B, c) - b0[c]) / DT)[i, i, i] for c in range(3)]
    assert np.abs(r[0] - A).max() <= 1e-10 * A
    assert np.abs(r[1]).max() == 0.0 and np.abs(r[2]).max() == 0.0
