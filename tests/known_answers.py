"""Known answers of the reference's verification routines, shared by the
CPU tests of the oracle and the GPU tests of the library.

* ``shercliff`` -- the fully developed MHD duct profile with insulating
  walls (profile_funcs.f90:65-138, shercliff_profile, and its coefficient
  shercliff_coeff :140-156, d_B = 0): Planas, Badia & Codina (2011), the
  series over alpha_k = (k + 1/2) pi / L, k = 0..1000.  The result variable
  starts at zero here (the reference accumulates into an uninitialised
  function result; its SH_profile variant zeroes it).
* ``hunt`` -- the same duct with perfectly conducting Hartmann walls
  (y = +-a, normal to B0) and insulating side walls (profile_funcs.f90:
  147-193, hunt_profile, and hunt_coeff :131-145).
* ``duct_steady`` -- runs a backend's MHD step (the B form with the
  constrained-transport induction source, finite Rem) on the square duct to
  its steady state, where it must reproduce the Shercliff profile (walls
  insulating: pseudo-vacuum BCs) or the Hunt profile (``walls="hunt"``: the
  induced field's BCs of a perfectly conducting Hartmann wall, B_y = 0 and
  d(B_x, B_z)/dn = 0 on y = +-a) at second order in the mesh spacing.
* ``taylor_green`` -- the decaying Taylor-Green vortex of
  GF_distributions.f90:720-769 (u = cos x sin y F, v = -sin x cos y F,
  F = exp(-2 t / Re)) with the BCs of init_U_BCs.f90:107-124 (Neumann /
  Dirichlet pairs on the x and y walls), on [0, pi]^2 x [0, 1] periodic in
  z; returns the max-norm error of (u, v) after T.
"""
from __future__ import annotations

import math

import numpy as np

from moons_b200 import capi as G
from moons_b200 import configs
from moons_b200 import mesh_gen as mg


def shercliff(x, y, Ha: float, Re: float, a: float = 1.0, b: float = 1.0, terms: int = 1000):
    L = b / a
    X, Y = np.meshgrid(np.asarray(x, float), np.asarray(y, float), indexing="ij")
    eta = Y / a
    w = np.zeros_like(X)

    def coeff(r1k, r2k):  # shercliff_coeff with d_B = 0
        A = (1.0 - np.exp(-2.0 * r2k)) / (1.0 + np.exp(-2.0 * r2k))
        B = (np.exp(-r1k * (1.0 - eta)) + np.exp(-r1k * (1.0 + eta))) / 2.0
        D = (1.0 - np.exp(-2.0 * (r1k + r2k))) / (1.0 + np.exp(-2.0 * r2k))
        return A * B / D

    for k in range(terms + 1):
        al = (k + 0.5) * math.pi / L
        N = math.sqrt(Ha ** 2 + 4.0 * al ** 2)
        r1, r2 = 0.5 * (Ha + N), 0.5 * (-Ha + N)
        w += 2.0 * (-1.0) ** k * np.cos(al * X / a) / (L * al ** 3) * (1.0 - coeff(r1, r2) - coeff(r2, r1))
    # w / mu * (-dpdz) * a^2 with mu = 1/Re and dp/dz = -1
    return w * Re * a ** 2


def hunt(x, y, Ha: float, Re: float, a: float = 1.0, b: float = 1.0, terms: int = 1000):
    L = b / a
    X, Y = np.meshgrid(np.asarray(x, float), np.asarray(y, float), indexing="ij")
    eta = Y / a
    w = np.zeros_like(X)

    def coeff(r1k, r2k, N):  # hunt_coeff
        return (r2k / N) * (np.exp(-r1k * (1.0 - eta)) + np.exp(-r1k * (1.0 + eta))) / (1.0 + np.exp(-2.0 * r1k))

    for k in range(terms + 1):
        al = (k + 0.5) * math.pi / L
        N = math.sqrt(Ha ** 2 + 4.0 * al ** 2)
        r1, r2 = 0.5 * (Ha + N), 0.5 * (-Ha + N)
        w += 2.0 * (-1.0) ** k * np.cos(al * X / a) / (L * al ** 3) * (1.0 - coeff(r1, r2, N) - coeff(r2, r1, N))
    return w * Re * a ** 2


def _hunt_duct(*args, **kw):
    """configs.duct with conducting Hartmann walls (y) and insulating side
    walls (x) for the induced field."""
    mom, ind, prm, init = configs.duct(*args, **kw)
    P, D, N = G.PERIODIC, G.DIRICHLET, G.NEUMANN
    types = ([N, N, N, N, P, P], [D, D, D, D, P, P], [D, D, N, N, P, P])
    for c in range(3):
        prm.bc_B[c] = G.bc_spec(types[c], order=configs.ORDER_PZ)
    return mom, ind, prm, init


def duct_steady(backend, n: int, beta: float = 1.05, Ha: float = 5.0, Re: float = 1.0, Rem: float = 1.0,
                dt: float = 0.01, max_steps: int = 1000, chunk: int = 50, settle: float = 1e-11,
                walls: str = "insulating"):
    """Relative max-norm error of the steady streamwise velocity against the
    Shercliff series (insulating walls) or the Hunt series (walls="hunt"),
    and the number of steps taken."""
    kw = dict(nx=n, ny=n, nz=4, Re=Re, Ha=Ha, Rem=Rem, dt=dt, n_wall=0, noise=0.0, beta=beta)
    builder = _hunt_duct if walls == "hunt" else configs.duct
    sim = configs.make(backend, builder, seed=0, tol=1e-12, **kw)
    prev, steps = None, 0
    while steps < max_steps:
        sim.step(chunk)
        steps += chunk
        w = sim.download(G.MHD_U, 2)
        if prev is not None and np.abs(w - prev).max() <= settle * np.abs(w).max():
            break
        prev = w.copy()
    mom = configs.duct(**kw)[0]
    hc = [0.5 * (h[1:] + h[:-1]) for h in mom]
    wa = (hunt if walls == "hunt" else shercliff)(hc[0][1:-1], hc[1][1:-1], Ha, Re)
    wn = w[1:-1, 1:-1, 2]
    return float(np.abs(wn - wa).max() / np.abs(wa).max()), steps


def taylor_green(backend, n: int, dt: float, T: float = 0.2, Re: float = 10.0, nz: int = 4) -> float:
    hx = mg.add_ghost_nodes(mg.uniform(0.0, math.pi, n))
    hz = mg.add_ghost_nodes(mg.uniform(0.0, 1.0, nz))
    hn = (hx, hx.copy(), hz)
    prm = G.MHDParams()
    prm.dt = dt
    prm.induction = G.IND_OFF
    configs._coeffs(prm, Re, 0.0, 1.0, False)
    for name in ("isp_U", "isp_p", "isp_B", "isp_phi"):
        setattr(prm, name, G.isp(5000, 1e-10, 1e-12, 1))
    D, N, P = G.DIRICHLET, G.NEUMANN, G.PERIODIC
    prm.bc_U[0] = G.bc_spec([N, N, D, D, P, P], order=configs.ORDER_PZ)
    prm.bc_U[1] = G.bc_spec([D, D, N, N, P, P], order=configs.ORDER_PZ)
    prm.bc_U[2] = G.bc_spec([D, D, D, D, P, P], order=configs.ORDER_PZ)
    prm.bc_p = G.bc_spec([N, N, N, N, P, P], order=configs.ORDER_PZ, all_neumann=True)
    for c in range(3):
        prm.bc_B[c] = G.bc_spec([D, D, D, D, P, P], order=configs.ORDER_PZ)
    prm.bc_phi = G.bc_spec([D, D, D, D, P, P], order=configs.ORDER_PZ)
    prm.prescribed_Ustar = 1
    prm.prescribed_Bstar = 1
    m = backend.Mesh(*hn)
    sim = backend.MHD(m, m, prm)
    hc = [0.5 * (h[1:] + h[:-1]) for h in hn]
    ones_z = np.ones(len(hc[2]))[None, None, :]

    def exact(t):
        F = math.exp(-2.0 / Re * t)
        u = np.cos(hn[0])[:, None, None] * np.sin(hc[1])[None, :, None] * F * ones_z
        v = -np.sin(hc[0])[:, None, None] * np.cos(hn[1])[None, :, None] * F * ones_z
        return u, v

    u, v = exact(0.0)
    sim.upload(G.MHD_U, 0, u)
    sim.upload(G.MHD_U, 1, v)
    sim.upload(G.MHD_U, 2, np.zeros(sim.shape(G.MHD_U, 2)))
    for c in range(3):
        sim.upload(G.MHD_B0, c, np.zeros(sim.shape(G.MHD_B0, c)))
        sim.upload(G.MHD_SIGMA_INV, c, np.ones(sim.shape(G.MHD_SIGMA_INV, c)))
    sim.init()
    ns = int(round(T / dt))
    sim.step(ns)
    ua, va = exact(ns * dt)
    I = (slice(1, -1),) * 3
    return float(max(np.abs(sim.download(G.MHD_U, 0) - ua)[I].max(),
                     np.abs(sim.download(G.MHD_U, 1) - va)[I].max()))


def grad_lap_commute(mod, backend, kind: str, n: int, seed: int = 5):
    """max over the three face components of |grad(lap phi) - lap(grad phi)|
    relative to |grad(lap phi)|, on the faces two or more cells from the
    boundary (operator_commute_test.f90:52-93); ``mod`` holds the operator
    functions (grad, lap_centered) of ``backend``."""
    from tests.common import coords
    hs = [coords(kind, n + 2 * i, 0.0, 1.0 + 0.3 * i) for i in range(3)]
    m = backend.Mesh(*hs)
    rng = np.random.default_rng(seed)
    phi = m.field(G.CC)
    a = np.zeros(phi.shape)
    a[1:-1, 1:-1, 1:-1] = rng.standard_normal(tuple(s - 2 for s in phi.shape))
    phi.upload(a)
    lp = m.field(G.CC)
    mod.lap_centered(lp, phi)
    LG = [m.field(d) for d in (G.FX, G.FY, G.FZ)]
    mod.grad(*LG, lp)
    gp = [m.field(d) for d in (G.FX, G.FY, G.FZ)]
    mod.grad(*gp, phi)
    GL = [m.field(d) for d in (G.FX, G.FY, G.FZ)]
    for o, i in zip(GL, gp):
        mod.lap_centered(o, i)
    I = (slice(2, -2),) * 3
    err = 0.0
    for d in range(3):
        x, y = GL[d].download()[I], LG[d].download()[I]
        err = max(err, float(np.abs(x - y).max() / np.abs(y).max()))
    return err
