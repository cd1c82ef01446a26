"""Case presets: the reference's compiled-in sim_params for the benchmark cases.

Each builder returns ``(mesh_mom_coords, mesh_ind_coords, params, init)``:
coordinates with ghost nodes (x, y, z), the C-ABI parameter struct and a
callable ``init(mhd, rng)`` that uploads the initial fields (seeded noise,
applied field, conductivity).  The same builder drives the CUDA library and
the CPU oracle, so both see identical inputs.

* ``ldc``  -- 3D MHD lid-driven cavity (sim_params_default_MHD_LDC_Sergey_uniform:
  LDC_at_ymax lid, Neumann pressure, uniform B0, solve_method 6), with the
  low-Rem electric-potential induction form or the reference's B form.
* ``duct`` -- fully developed MHD duct (sim_params_default_MHD_Shercliff:
  periodic streamwise, mean pressure gradient, finite Rem, solve_method 6),
  Roberts two-sided clustering (robertsBoth, beta=1.05) across, and a
  conducting wall layer in the induction mesh (MD_sigma/MD_fluid split).
* ``full_bc`` -- the reference's full_BC case (sim_params_default_full_BC):
  lid-driven MHD cavity on the mesh bank's full_BC_w_vacuum_3D meshes
  (boundary-layer clustered fluid, thin conducting walls, vacuum out to
  |x| = 7), finite Rem, B form, sigma = 1 in fluid and walls and
  sig_local_over_sig_f outside them.
"""
from __future__ import annotations

import math

import numpy as np

from . import capi as G
from . import mesh_bank as mb
from . import mesh_gen as mg

ORDER_LDC = (5, 6, 1, 2, 3, 4)   # get_apply_BC_order for periodic_dir = 0 (sim_params_aux.f90:41)
ORDER_PZ = (1, 2, 3, 4, 5, 6)    # get_apply_BC_order for periodic z       (sim_params_aux.f90:48)


def _isp(iter_max, tol_rel, tol_abs=1e-15, nskip=1):
    return G.isp(iter_max, tol_rel, tol_abs, nskip)


def _coeffs(prm, Re, Ha, Rem, finite_Rem):
    # var_set_extend.f90:55-86 with alpha = 1 (backward Euler) -> beta = 0
    N = Ha ** 2 / Re
    prm.coeff_implicit_U = -(1.0 / Re)                       # -coeff_natural*alpha, coeff_natural = 1/Re
    prm.coeff_implicit_B = -(-1.0 / Rem)                     # coeff_natural = -1/Rem
    prm.scale_advection_U = -1.0
    prm.scale_diffusion_U = 0.0                              # coeff_natural*beta
    prm.scale_JxB = N
    prm.scale_advection_B = 1.0
    prm.scale_diffusion_B = -0.0                             # -beta
    prm.scale_current = 1.0 / Rem
    prm.finite_Rem = 1 if finite_Rem else 0
    return N


def ldc(n: int = 32, Re: float = 400.0, Ha: float = 10.0, dt: float = 1e-3, induction: int = G.IND_POTENTIAL,
        Rem: float = 1.0, tol: float = 1e-10, noise: float = 1e-6, iter_max: int = 20000):
    h = mg.add_ghost_nodes(mg.uniform(0.0, 1.0, n))
    coords = (h, h.copy(), h.copy())
    prm = G.MHDParams()
    prm.dt = dt
    prm.induction = induction
    _coeffs(prm, Re, Ha, Rem, False)
    prm.mpg_dir = 0
    prm.mpg_scale = 0.0
    for name in ("isp_U", "isp_p", "isp_B", "isp_phi"):
        setattr(prm, name, _isp(iter_max, tol))
    for c in range(3):
        vals = [0.0] * 6
        if c == 0:
            vals[3] = 1.0  # LDC_at_ymax: init(U%x%BF(1)%BCs,1.0,4)
        prm.bc_U[c] = G.bc_spec([G.DIRICHLET] * 6, values=vals, order=ORDER_LDC)
        t = [G.DIRICHLET] * 6
        t[2 * c] = t[2 * c + 1] = G.NEUMANN  # pseudo_vacuum (init_B_BCs.f90:83-97)
        prm.bc_B[c] = G.bc_spec(t, order=ORDER_LDC)
    prm.bc_p = G.bc_spec([G.NEUMANN] * 6, order=ORDER_LDC, all_neumann=True)
    if induction == G.IND_POTENTIAL:
        # insulating walls: J.n = 0 -> homogeneous Neumann for the potential
        prm.bc_phi = G.bc_spec([G.NEUMANN] * 6, order=ORDER_LDC, all_neumann=True)
    else:
        prm.bc_phi = G.bc_spec([G.DIRICHLET] * 6, order=ORDER_LDC)  # init_phi_BCs default
    prm.prescribed_Ustar = 1
    prm.prescribed_Bstar = 1

    def init(sim, rng):
        for c in range(3):
            s = sim.shape(G.MHD_U, c)
            sim.upload(G.MHD_U, c, rng.normal(0.0, noise, s))
            b0 = np.zeros(sim.shape(G.MHD_B0, c))
            if c == 1:
                b0[:] = 1.0  # uniform_B_field dir=2
            sim.upload(G.MHD_B0, c, b0)
            sim.upload(G.MHD_SIGMA_INV, c, np.ones(sim.shape(G.MHD_SIGMA_INV, c)))

    return coords, coords, prm, init


def duct(nx: int = 64, ny: int = 64, nz: int = 256, Re: float = 1000.0, Ha: float = 100.0, dt: float = 5e-4,
         beta: float = 1.05, n_wall: int = 4, t_wall: float = 1.0, sigma_wall: float = 0.01, Lz: float = 8.0,
         Rem: float = 1.0, tol: float = 1e-10, noise: float = 1e-4, iter_max: int = 20000):
    """Streamwise z (periodic), field along y, walls normal to x and y."""
    hx = mg.roberts_both(-1.0, 1.0, nx, beta)
    hy = mg.roberts_both(-1.0, 1.0, ny, beta)
    hz = mg.uniform(0.0, Lz, nz)
    mom = (mg.add_ghost_nodes(hx), mg.add_ghost_nodes(hy), mg.add_ghost_nodes(hz))
    if n_wall > 0:
        w = t_wall / n_wall
        ext = lambda h: np.concatenate([h[0] - w * np.arange(n_wall, 0, -1), h, h[-1] + w * np.arange(1, n_wall + 1)])
        ind = (mg.add_ghost_nodes(ext(hx)), mg.add_ghost_nodes(ext(hy)), mg.add_ghost_nodes(hz))
        off = (n_wall, n_wall, 0)
    else:
        ind = mom
        off = (0, 0, 0)
    prm = G.MHDParams()
    prm.dt = dt
    prm.induction = G.IND_B
    _coeffs(prm, Re, Ha, Rem, True)
    prm.mpg_dir = 3
    prm.mpg_scale = 1.0  # SP%MT%mean_pressure_grad scale (Shercliff preset), dp/dz = -1
    for name in ("isp_U", "isp_p", "isp_B", "isp_phi"):
        setattr(prm, name, _isp(iter_max, tol))
    P, D, N = G.PERIODIC, G.DIRICHLET, G.NEUMANN
    for c in range(3):
        prm.bc_U[c] = G.bc_spec([D, D, D, D, P, P], order=ORDER_PZ)
        t = [D, D, D, D, P, P]
        if c < 2:
            t[2 * c] = t[2 * c + 1] = N  # pseudo_vacuum outside the wall layer
        prm.bc_B[c] = G.bc_spec(t, order=ORDER_PZ)
    prm.bc_p = G.bc_spec([N, N, N, N, P, P], order=ORDER_PZ, all_neumann=True)
    prm.bc_phi = G.bc_spec([D, D, D, D, P, P], order=ORDER_PZ)
    prm.prescribed_Ustar = 1
    prm.prescribed_Bstar = 1
    for d in range(3):
        prm.ind_offset[d] = off[d]

    def init(sim, rng):
        for c in range(3):
            sim.upload(G.MHD_U, c, rng.normal(0.0, noise, sim.shape(G.MHD_U, c)))
            b0 = np.zeros(sim.shape(G.MHD_B0, c))
            if c == 1:
                b0[:] = 1.0
            sim.upload(G.MHD_B0, c, b0)
        # sigma^-1 on edges: 1 inside the closed fluid box, 1/sigma_wall in the wall layer
        hn = ind
        lo = [mom[d][1] for d in range(3)]
        hi = [mom[d][-2] for d in range(3)]
        hc = [0.5 * (h[1:] + h[:-1]) for h in hn]
        tol_ = 1e-12
        for c in range(3):  # edge along c: CC along c, N elsewhere
            axes = [hc[d] if d == c else hn[d] for d in range(3)]
            inside = [(a >= lo[d] - tol_) & (a <= hi[d] + tol_) if d < 2 else np.ones_like(a, bool)
                      for d, a in enumerate(axes)]
            m3 = inside[0][:, None, None] & inside[1][None, :, None] & inside[2][None, None, :]
            si = np.where(m3, 1.0, 1.0 / sigma_wall)
            sim.upload(G.MHD_SIGMA_INV, c, si)

    return mom, ind, prm, init


def at_scale(nx: int = 128, ny: int = 128, nz: int = 256, **kw):
    """Full solver at scale: finite magnetic Reynolds number with constrained
    transport (the B form), 256 x 128 x 128 cells (streamwise z uniform, the
    cross-section Roberts-stretched), Re = 1000, Ha = 500, Rem = 10,
    dt = 2e-4, seeded N(0, 1e-3) velocity, insulating walls (no wall layer).
    The duct geometry and BCs of ``duct``."""
    args = dict(Re=1000.0, Ha=500.0, Rem=10.0, dt=2e-4, noise=1e-3, n_wall=0)
    args.update(kw)
    return duct(nx=nx, ny=ny, nz=nz, **args)


def ldc_energy(n: int = 16, Pe: float = 100.0, Gr_Re2: float = 10.0, heating: float = 0.5,
               solve_method_T: int = 3, tol: float = 1e-10, KE_diffusion: float = 0.0,
               viscous_dissipation: float = 0.0, joule_heating: float = 0.0, **kw):
    """The lid-driven cavity with the energy equation: T = 1 on the x-min
    wall, 0 on x-max, insulated elsewhere; conductivity on the faces varying
    by +-20% (seeded); gravity -y; advection scale 1 (S += -div(u T)),
    diffusion by the implicit nrg_diffusion PCG (solve_method 3 and 4,
    coefficient -1/Pe), explicitly (solve_method 1 and 2, scale 1/Pe), or
    half and half (solve_method 5 with three RK stages: the explicit part
    goes into L and is weighed by alpha, the implicit by beta, each summing
    to 1/2 over the stages); volumetric heating
    (add_volumetric_heating_Nuclear) and buoyancy Gr/Re^2 in momentum;
    optionally the KE-diffusion, viscous-dissipation and Joule-heating
    sources with the given scales (sigma^-1 at cell centres then 1 + 0.5 x,
    so the Joule term does not vanish as it would with the reference's
    never-set ind%sigmaInv_CC)."""
    mom, ind, prm, init0 = ldc(n=n, tol=tol, **kw)
    prm.energy = 1
    prm.solve_method_T = solve_method_T
    prm.coeff_implicit_T = -1.0 / Pe
    prm.scale_advection_T = 1.0
    prm.scale_diffusion_T = 0.0 if solve_method_T in (3, 4) else 1.0 / Pe
    prm.scale_heating_T = heating
    prm.scale_buoyancy = Gr_Re2
    prm.isp_T = _isp(5000, tol)
    prm.scale_KE_diffusion_T = KE_diffusion
    prm.scale_viscous_dissipation_T = viscous_dissipation
    prm.scale_joule_heating_T = joule_heating
    D, Nn = G.DIRICHLET, G.NEUMANN
    prm.bc_T = G.bc_spec([D, D, Nn, Nn, Nn, Nn], values=[1.0, 0.0, 0.0, 0.0, 0.0, 0.0], order=ORDER_LDC)

    def init(sim, rng):
        init0(sim, rng)
        for c in range(3):
            sim.upload(G.MHD_KT, c, 1.0 + 0.2 * rng.uniform(-1.0, 1.0, sim.shape(G.MHD_KT, c)))
            g = np.zeros(sim.shape(G.MHD_GRAVITY, c))
            if c == 1:
                g[:] = -1.0
            sim.upload(G.MHD_GRAVITY, c, g)
        if joule_heating != 0.0:
            hx = ind[0]
            xc = 0.5 * (hx[1:] + hx[:-1])
            sic = np.ones(sim.shape(G.MHD_SIGMA_INV_CC)) * (1.0 + 0.5 * xc)[:, None, None]
            sim.upload(G.MHD_SIGMA_INV_CC, 0, sic)

    return mom, ind, prm, init


def sigma_inv_edges(ind, sigma, sig_local: float):
    """1/sigma on the induction mesh's edges as set_sigma_inv_VF sets it
    (solvers/induction/induction_aux.f90:178-194): 1/sig_local_over_sig_f
    everywhere, then 1 embedded over the conductor mesh's physical overlap
    (edge along c: the shared cells along c, the shared nodes, boundary nodes
    included, along the other two directions)."""
    rng = mg.sub_domain_ranges(sigma, ind)
    out = []
    for c in range(3):
        shape = tuple(len(ind[d]) - 1 if d == c else len(ind[d]) for d in range(3))
        si = np.full(shape, 1.0 / sig_local)
        sl = tuple(slice(*rng[d][0]) if d == c else slice(*rng[d][1]) for d in range(3))
        si[sl] = 1.0
        out.append(si)
    return out


def full_bc(N: int = 80, N_w: int = 9, vacuum: bool = True, Re: float = 2000.0, N_stuart: float = 5.0,
            Rem: float = 2000.0, dt: float = 2.5e-3, sig_local: float = 1e-3, tol: float = 1e-6,
            tol_abs: float = 1e-13, iter_max=(5, 20, 20, 20), noise: float = 0.0, mqp=None):
    """sim_params_default_full_BC: Re = 2000, N = 5 (Ha = sqrt(N Re) = 100),
    Rem = 2000 with finite_Rem, dt = 2.5e-3, the lid-driven cavity
    (U preset 1: LDC_at_ymax), B0 = 1 along z (uniform_B0_dir = 3), B = 0 on
    the induction mesh's outer boundary (B preset 0: Dirichlet), Neumann
    pressure, Dirichlet potential, prescribed BCs on U* and B*, solve
    method 6, PCG limits U 5, p 20, B 20, phi 20 iterations at tol_rel 1e-6,
    tol_abs 1e-13.  Meshes from the mesh bank (full_BC_w_vacuum_3D, or
    full_BC_n_vacuum_3D with ``vacuum=False``) at N and N_w; the fluid sits
    in the induction mesh at the offset the sub-domain overlap finds.
    ``iter_max`` = (U, p, B, phi)."""
    Ha = math.sqrt(N_stuart * Re)
    ms = (mb.full_bc_w_vacuum_3d if vacuum else mb.full_bc_n_vacuum_3d)(N, N_w, mqp)
    m = mb.generate(ms, Re, Ha)
    off = mg.sub_domain_offset(m.mom, m.ind)
    prm = G.MHDParams()
    prm.dt = dt
    prm.induction = G.IND_B
    _coeffs(prm, Re, Ha, Rem, True)
    prm.mpg_dir = 0
    prm.mpg_scale = 0.0
    for name, it in zip(("isp_U", "isp_p", "isp_B", "isp_phi"), iter_max):
        setattr(prm, name, G.isp(it, tol, tol_abs, 1))
    for c in range(3):
        vals = [0.0] * 6
        if c == 0:
            vals[3] = 1.0  # LDC_at_ymax
        prm.bc_U[c] = G.bc_spec([G.DIRICHLET] * 6, values=vals, order=ORDER_LDC)
        prm.bc_B[c] = G.bc_spec([G.DIRICHLET] * 6, order=ORDER_LDC)
    prm.bc_p = G.bc_spec([G.NEUMANN] * 6, order=ORDER_LDC, all_neumann=True)
    prm.bc_phi = G.bc_spec([G.DIRICHLET] * 6, order=ORDER_LDC)
    prm.prescribed_Ustar = 1
    prm.prescribed_Bstar = 1
    for d in range(3):
        prm.ind_offset[d] = off[d]
    si = sigma_inv_edges(m.ind, m.sigma, sig_local)

    def init(sim, rng):
        for c in range(3):
            s = sim.shape(G.MHD_U, c)
            sim.upload(G.MHD_U, c, rng.normal(0.0, noise, s) if noise > 0 else np.zeros(s))
            b0 = np.zeros(sim.shape(G.MHD_B0, c))
            if c == 2:
                b0[:] = 1.0  # uniform_B_field dir = 3
            sim.upload(G.MHD_B0, c, b0)
            sim.upload(G.MHD_SIGMA_INV, c, si[c])

    return m.mom, m.ind, prm, init


def make(backend, builder, *args, seed: int = 0, prec_poisson: int = 0, unets=None, meshes=None,
         solve_method_U: int = 0, solve_method_B: int = 0, **kw):
    """Create meshes + the MHD object on ``backend`` (moons_b200.capi or the
    oracle module) from a builder, upload the seeded initial state and init.
    ``prec_poisson`` selects the pressure/potential preconditioner (0: the
    reference's Jacobi prec_Lap; capi.PREC_MG / PREC_MG_MIXED: multigrid;
    PREC_FD: the direct solve; PREC_UNET_MG: learned + mixed, with
    ``unets`` = (pressure net, potential net) built on ``meshes`` = (fluid
    mesh, induction mesh), which the simulation then uses).
    ``solve_method_U`` / ``solve_method_B`` pick the momentum / induction
    time scheme (0 or 6: Euler_time_AB2_sources, 5: Euler_time_Euler_sources,
    7: O2_BDF_time_AB2_sources; time_marching_methods.f90:47-150)."""
    mom, ind, prm, init = builder(*args, **kw)
    prm.prec_poisson = prec_poisson
    prm.solve_method_U = solve_method_U
    prm.solve_method_B = solve_method_B
    if meshes is not None:
        mm, mi = meshes
    else:
        mm = backend.Mesh(*mom)
        mi = mm if ind is mom else backend.Mesh(*ind)
    sim = backend.MHD(mm, mi, prm)
    if unets is not None:
        for which, net in enumerate(unets):
            if net is not None:
                sim.set_unet(which, net)
    init(sim, np.random.default_rng(seed))
    sim.init()
    return sim


def sigma_shell(n: int = 128, shell: int = 4, seed: int = 0):
    """Mixed-precision Poisson case: div(sigma grad phi) = div(u x B) on the
    uniform unit cube with n^3 cells, sigma = 1 inside and one seeded draw of
    10^U(-3,3) in a `shell`-cell layer along every wall; u and B i.i.d.
    N(0,1) per face; insulating walls (Neumann everywhere), so the solver
    removes the right-hand side's mean (all_neumann).

    Returns (coords, sigma_faces, E_faces): node coordinates with ghosts,
    sigma on the x/y/z faces (mean of the two adjacent cells, the reference's
    cell-to-face interpolation), and E = u x B on the faces (the other
    components of u and B brought to each face by the mean of the four
    surrounding faces, face2Face_no_diag), all as Fortran-layout arrays with
    ghosts.  div(E) is formed by the library's own divergence."""
    rng = np.random.default_rng(seed)
    h = mg.add_ghost_nodes(mg.uniform(0.0, 1.0, n))
    coords = (h, h.copy(), h.copy())
    sc = n + 2
    sig_c = np.ones((sc, sc, sc))
    s_wall = 10.0 ** rng.uniform(-3.0, 3.0)
    idx = np.arange(sc)
    inner = (idx >= 1 + shell) & (idx <= n - shell)
    ins = inner[:, None, None] & inner[None, :, None] & inner[None, None, :]
    sig_c[~ins] = s_wall
    sig_f = []
    for d in range(3):
        shp = [sc, sc, sc]
        shp[d] = sc + 1
        f = np.ones(shp)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        mid = [slice(None)] * 3
        lo[d] = slice(0, sc - 1)
        hi[d] = slice(1, sc)
        mid[d] = slice(1, sc)
        f[tuple(mid)] = 0.5 * (sig_c[tuple(lo)] + sig_c[tuple(hi)])
        sig_f.append(f)
    # u, B on faces
    def faces():
        out = []
        for d in range(3):
            shp = [sc, sc, sc]
            shp[d] = sc + 1
            out.append(rng.standard_normal(shp))
        return out
    u, B = faces(), faces()

    def to_face(a, src, dst):
        # mean of the four src-faces around each dst-face (interior entries)
        shp = [sc, sc, sc]
        shp[dst] = sc + 1
        out = np.zeros(shp)
        # cell-centre value of the src component: mean of its two faces
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[src] = slice(0, sc)
        hi[src] = slice(1, sc + 1)
        cc = 0.5 * (a[tuple(lo)] + a[tuple(hi)])
        # cell centre -> dst faces: mean of the two neighbouring cells
        l2 = [slice(None)] * 3
        h2 = [slice(None)] * 3
        m2 = [slice(None)] * 3
        l2[dst] = slice(0, sc - 1)
        h2[dst] = slice(1, sc)
        m2[dst] = slice(1, sc)
        out[tuple(m2)] = 0.5 * (cc[tuple(l2)] + cc[tuple(h2)])
        return out

    E = []
    for d in range(3):
        a, b = (d + 1) % 3, (d + 2) % 3
        E.append(to_face(u[a], a, d) * to_face(B[b], b, d) - to_face(u[b], b, d) * to_face(B[a], a, d))
    return coords, sig_f, E
