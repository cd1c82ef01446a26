"""Mesh generation of the reference (moons_b200.mesh_gen, moons_b200.mesh_bank):
the coordinate distributions, the mesh-quality search, the Roberts parameter
matched to an end spacing, grid extensions, the generic generator, the mesh
bank presets and the sub-domain overlap that places the fluid mesh inside
the induction mesh."""
import math

import numpy as np
import pytest

from moons_b200 import configs
from moons_b200 import mesh_bank as mb
from moons_b200 import mesh_gen as mg

AUTO = mg.MeshQuality(True, 2.0, 50)


def ratios(h):
    d = np.diff(h)
    return np.maximum(d[1:] / d[:-1], d[:-1] / d[1:])


# ---- distributions ---------------------------------------------------------------

@pytest.mark.parametrize("n", [1, 2, 7, 40])
def test_uniform_and_linspace(n):
    h = mg.uniform(-1.0, 3.0, n)
    assert len(h) == n + 1 and h[0] == -1.0
    assert np.allclose(np.diff(h), 4.0 / n, rtol=0, atol=1e-14)
    assert np.array_equal(h, mg.linspace(-1.0, 3.0, n))


def test_uniform_edge_cases():
    assert np.array_equal(mg.uniform(2.0, 2.0, 0), [2.0])
    with pytest.raises(ValueError):
        mg.uniform(0.0, 1.0, 0)
    with pytest.raises(ValueError):
        mg.uniform(0.0, 1.0, -1)
    assert np.array_equal(mg.uniform_left(1.0, 0.0, 0), [1.0])
    with pytest.raises(ValueError):
        mg.uniform_left(1.0, 0.5, 0)


def test_uniform_left_right():
    r = mg.uniform_right(1.0, 0.25, 4)
    l = mg.uniform_left(1.0, 0.25, 4)
    assert np.allclose(r, [1.0, 1.25, 1.5, 1.75, 2.0])
    assert np.allclose(l, [0.0, 0.25, 0.5, 0.75, 1.0])
    assert l[-1] == 1.0 and r[0] == 1.0


@pytest.mark.parametrize("beta", [1.001, 1.05, 1.5, 10.0])
@pytest.mark.parametrize("n", [4, 17, 64])
def test_roberts_families(beta, n):
    R = mg.roberts_right(0.0, 2.0, n, beta)
    L = mg.roberts_left(0.0, 2.0, n, beta)
    B = mg.roberts_both(0.0, 2.0, n, beta)
    for h in (R, L, B):
        assert len(h) == n + 1
        assert abs(h[0]) < 1e-15 and abs(h[-1] - 2.0) < 1e-14
        assert np.all(np.diff(h) > 0)
    # transformation1 is the mirror image of transformation2 with alpha = 0
    assert np.allclose(L, 2.0 - R[::-1], rtol=0, atol=1e-13)
    # clustering: right fine at hmax, left fine at hmin, both symmetric
    assert np.all(np.diff(np.diff(R)) <= 1e-15) and np.all(np.diff(np.diff(L)) >= -1e-15)
    assert np.allclose(np.diff(B), np.diff(B)[::-1], rtol=1e-10, atol=1e-14)


def test_cluster_distribution():
    h = mg.cluster(0.0, 1.0, 40, 0.3, 4.0)
    assert abs(h[0]) < 1e-14 and abs(h[-1] - 1.0) < 1e-12
    d = np.diff(h)
    assert np.all(d > 0)
    # finest cells around yc
    i = int(np.argmin(d))
    assert abs(0.5 * (h[i] + h[i + 1]) - 0.3) < 0.05


# ---- boundary-layer parameters ---------------------------------------------------

def test_boundary_layer_parameters():
    assert mg.roberts_bl_1d(0.1, 2.0) == pytest.approx((1 - 0.05) ** -0.5, rel=1e-15)
    assert mg.roberts_bl_1d(1.99, 2.0) == 1000.0     # delta >= 0.99 h
    Re, Ha = 1000.0, 50.0
    r = mg.reynolds_bl_1d(Re, -1.0, 1.0)
    h = mg.hartmann_bl_1d(Ha, -1.0, 1.0)
    assert r == pytest.approx((1 - 1 / math.sqrt(Re)) ** -0.5)
    assert h == pytest.approx((1 - 1 / Ha) ** -0.5)
    assert mg.re_ha_bl_1d(Re, Ha, -1.0, 1.0) == min(r, h)
    with pytest.raises(ValueError):
        mg.re_ha_bl_1d(Re, 0.0, -1.0, 1.0)
    with pytest.raises(ValueError):
        mg.re_ha_bl_1d(0.0, Ha, -1.0, 1.0)


# ---- Roberts parameter matched to an end spacing ---------------------------------

@pytest.mark.parametrize("n,dh", [(5, 0.01), (10, 0.01), (20, 0.02), (40, 0.001)])
def test_beta_match_end_spacing(n, dh):
    b = mg.beta_dh_small(0.0, 1.0, n, dh)
    h = mg.roberts_right(0.0, 1.0, n, b)
    assert mg.last_match_error is None
    assert abs((h[-1] - h[-2]) - dh) < 1e-13
    b = mg.beta_dh_both(0.0, 1.0, n, dh)
    h = mg.roberts_both(0.0, 1.0, n, b)
    assert mg.last_match_error is None
    assert abs((h[-1] - h[-2]) - dh) < 1e-13 and abs((h[1] - h[0]) - dh) < 1e-13


def test_beta_match_big_end():
    b = mg.beta_dh_big(0.0, 1.0, 10, 0.2)
    h = mg.roberts_right(0.0, 1.0, 10, b)
    assert mg.last_match_error is None
    assert abs((h[1] - h[0]) - 0.2) < 1e-13


def test_beta_match_falls_back_to_1p1():
    # a uniform end cell needs beta -> infinity: the iteration passes 1000
    # without converging and the reference falls back to beta = 1.1
    assert mg.beta_dh_big(0.0, 1.0, 5, 0.2) == 1.1
    assert mg.last_match_error is not None


# ---- mesh quality search -----------------------------------------------------------

def test_needs_more_points():
    q = mg.MeshQuality(True, 2.0, 5)
    assert not mg.needs_more_points([0.0, 1.0], q)
    assert not mg.needs_more_points([0.0, 1.0, 2.5], q)
    assert mg.needs_more_points([0.0, 1.0, 3.5], q)
    assert mg.MeshQuality().N_iter == 1 and q.N_iter == 6


def test_iterate_adds_points_until_the_ratio_holds():
    beta = 1.0005
    once = mg.roberts_both_iterate(-1.0, 1.0, 8, beta, mg.MeshQuality())
    assert len(once) == 9 and ratios(once).max() > 2.0
    h = mg.roberts_both_iterate(-1.0, 1.0, 8, beta, AUTO)
    assert ratios(h).max() <= 2.0
    n = len(h) - 1
    assert n > 8
    # the smallest count that satisfies it
    assert ratios(mg.roberts_both(-1.0, 1.0, n - 1, beta)).max() > 2.0
    with pytest.raises(ValueError):
        mg.roberts_both_iterate(-1.0, 1.0, 8, beta, mg.MeshQuality(True, 2.0, -1))  # N_iter = 0


# ---- grids and extensions ---------------------------------------------------------

def test_ghost_nodes():
    h = mg.add_ghost_nodes(np.array([0.0, 0.1, 0.3, 0.6]))
    assert np.allclose(h, [-0.1, 0.0, 0.1, 0.3, 0.6, 0.9])
    with pytest.raises(ValueError):
        mg.add_ghost_nodes(np.array([1.0]))


def test_uniform_extension_both_sides():
    g = mg.Grid()
    g.grid_roberts_b(-1.0, 1.0, 10, 1.05, 1, mg.MeshQuality())
    base = g.hn[0].copy()
    dh0, dh1 = base[2] - base[1], base[-2] - base[-3]
    g.ext_uniform(3, 1)
    h = g.hn[0]
    assert len(h) == len(base) + 6
    assert np.allclose(np.diff(h[1:5]), dh0) and np.allclose(np.diff(h[-5:-1]), dh1)
    assert np.array_equal(h[4:-4], base[1:-1])
    # ghosts mirror the end spacing
    assert h[1] - h[0] == pytest.approx(h[2] - h[1]) and h[-1] - h[-2] == pytest.approx(h[-2] - h[-3])


@pytest.mark.parametrize("kind", ["near", "far", "b", "c2f"])
def test_roberts_extensions_match_the_join(kind):
    q = mg.MeshQuality()
    g = mg.Grid()
    g.grid_roberts_b(-1.0, 1.0, 20, 1.02, 2, q)
    base = g.hn[1][1:-1].copy()
    dh_lo, dh_hi = base[1] - base[0], base[-1] - base[-2]
    # C2F puts the matched cell at the coarse end: it needs an end cell larger
    # than the uniform one (L / n), else the match falls back to beta = 1.1
    L, n = (0.1, 12) if kind == "c2f" else (0.5, 12)
    if kind == "near":
        g.ext_roberts_near(L, n, 2, q)
    elif kind == "far":
        g.ext_roberts_far(L, n, 2, q)
    elif kind == "b":
        g.ext_roberts_b(L, n, 2, q)
    else:
        g.ext_prep_roberts_c2f(L, n, 2, q)
        g.ext_app_roberts_c2f(L, n, 2, q)
    h = g.hn[1][1:-1]
    assert len(h) == len(base) + 2 * n
    assert h[0] == pytest.approx(-1.0 - L, abs=1e-14) and h[-1] == pytest.approx(1.0 + L, abs=1e-14)
    assert np.array_equal(h[n:-n], base)
    assert mg.last_match_error is None
    d = np.diff(h)
    if kind in ("near", "b", "c2f"):
        # the cell next to the base mesh has the base mesh's end size
        assert d[n - 1] == pytest.approx(dh_lo, rel=1e-10) and d[-n] == pytest.approx(dh_hi, rel=1e-10)
    if kind == "far":
        # the matched (small) cell sits at the far end
        assert d[0] == pytest.approx(dh_lo, rel=1e-10) and d[-1] == pytest.approx(dh_hi, rel=1e-10)


def test_extension_point_search_steps_by_two():
    # the reference's loop takes the point count of the last try (cells + 1)
    # before adding one, so searched extensions grow by two cells at a time
    g = mg.Grid()
    g.grid_roberts_b(-1.0, 1.0, 30, 1.001, 1, AUTO)
    n0 = len(g.hn[0])
    g.ext_prep_roberts_b(0.05, 4, 1, AUTO)
    added = len(g.hn[0]) - n0
    assert added >= 4 and (added - 4) % 2 == 0


def test_extension_errors():
    g = mg.Grid()
    with pytest.raises(ValueError):
        g.ext_uniform(2, 1)       # no base distribution yet
    g.grid_uniform(0.0, 1.0, 4, 1)
    with pytest.raises(ValueError):
        g.ext_app_uniform(0, 1)   # check_N


# ---- generic generator and mesh bank -----------------------------------------------

def test_generate_mesh_generic_segments():
    mp = mg.MeshParams(mg.MeshQuality())
    mp.add_base(mg.seg_1d(1, "grid_uniform", 4, 0.0, 1.0, 1.0))
    mp.add_base(mg.seg_1d(2, "grid_Roberts_B", 6, -1.0, 1.0, 1.0))
    mp.add_base(mg.seg_1d(3, "grid_uniform", 0, 0.0, 1.0, 1.0))   # no cells: skipped
    mp.add_base(mg.seg_1d(3, "grid_uniform", 2, 0.0, 1.0, 1.0))
    mp.add_ext(mg.seg_1d(1, "ext_app_uniform_IO", 2))
    g = mg.generate_mesh_generic(mp, 100.0, 10.0)
    assert g.cells() == (6, 6, 2)
    beta = mg.re_ha_bl_1d(100.0, 10.0, -1.0, 1.0)
    assert np.allclose(g.hn[1][1:-1], mg.roberts_both(-1.0, 1.0, 6, beta), rtol=0, atol=1e-15)
    bad = mg.MeshParams(mg.MeshQuality())
    bad.add_base(mg.seg_1d(1, "grid_spline", 4, 0.0, 1.0, 1.0))
    with pytest.raises(ValueError):
        mg.generate_mesh_generic(bad, 100.0, 10.0)


def test_mesh_bank_sergey_uniform_is_exact():
    m = mb.generate(mb.mhd_ldc_sergey_uniform(), 100.0, 10.0)
    for d in range(3):
        assert len(m.mom[d]) - 3 == 45 and len(m.ind[d]) - 3 == 67
        assert np.allclose(np.diff(m.ind[d]), 2.0 / 45, rtol=0, atol=1e-13)
        assert m.ind[d][1] == pytest.approx(-1.0 - 11 * 2.0 / 45, abs=1e-13)
    assert mg.sub_domain_offset(m.mom, m.ind) == (11, 11, 11)
    assert mg.sub_domain_offset(m.sigma, m.ind) == (11, 11, 11)


def test_mesh_bank_two_dimensional_presets():
    m = mb.generate(mb.hydro_ldc_ghia(), 400.0, 1.0)
    assert tuple(len(h) - 3 for h in m.mom) == (64, 64, 1)
    m = mb.generate(mb.bandaru(), 100.0, 10.0)
    assert tuple(len(h) - 3 for h in m.mom) == (130, 1, 130)
    assert m.mom[0][1] == 0.0 and m.mom[0][-2] == pytest.approx(2.0 * mb.PI)


@pytest.mark.parametrize("name", sorted(mb.PRESETS))
def test_every_preset_generates_nested_meshes(name):
    m = mb.generate(mb.PRESETS[name](), 2000.0, 100.0)
    for mesh in m:
        for h in mesh:
            assert np.all(np.diff(h) > 0)
    # the fluid sits inside the conductor, the conductor inside the induction mesh
    mg.sub_domain_offset(m.mom, m.sigma)
    mg.sub_domain_offset(m.sigma, m.ind)
    mg.sub_domain_offset(m.mom, m.ind)


def test_full_bc_w_vacuum_3d_layout():
    m = mb.generate(mb.full_bc_w_vacuum_3d(), 2000.0, 100.0)
    assert tuple(len(h) - 3 for h in m.mom) == (80, 85, 80)
    lo = [h[1] for h in m.ind]
    hi = [h[-2] for h in m.ind]
    # vacuum out to 7 on every side except the lid side's 6 + 1
    assert np.allclose(lo, [-7.0, -7.0, -7.0]) and np.allclose(hi, [7.0, 7.0, 7.0])
    fl = [(h[1], h[-2]) for h in m.mom]
    assert np.allclose(fl, [(-1.0, 1.0)] * 3)
    # the wall: 0.05 thick on five sides, none above the lid
    sg = [(h[1], h[-2]) for h in m.sigma]
    assert np.allclose(sg, [(-1.05, 1.05), (-1.05, 1.0), (-1.05, 1.05)])


# ---- overlaps and the conductivity of the vacuum case ------------------------------

def test_overlap_ranges():
    outer = mg.add_ghost_nodes(mg.uniform(-2.0, 2.0, 8))
    inner = mg.add_ghost_nodes(mg.uniform(-1.0, 1.0, 4))
    c = mg.c_overlap(inner, outer, p=1)
    n = mg.n_overlap(inner, outer, p=1)
    assert c.i1 == (2, 5) and c.i2 == (4, 7) and c.success and c.valid_range()
    assert n.i1 == (2, 6) and n.i2 == (4, 8)
    # total overlap (ghosts included): the inner ghost cells are outer cells too
    t = mg.c_overlap(inner, outer, p=0)
    assert t.i1 == (1, 6) and t.i2 == (3, 8)
    assert mg.sub_domain_offset([inner] * 3, [outer] * 3) == (2, 2, 2)
    far = mg.add_ghost_nodes(mg.uniform(5.0, 6.0, 2))
    assert not mg.is_overlap(far, inner)
    with pytest.raises(ValueError):
        mg.sub_domain_offset([far] * 3, [inner] * 3)


def test_sigma_inv_of_the_vacuum_case():
    m = mb.generate(mb.full_bc_w_vacuum_3d(8, 3), 2000.0, 100.0)
    si = configs.sigma_inv_edges(m.ind, m.sigma, 1e-3)
    rng = mg.sub_domain_ranges(m.sigma, m.ind)
    for c in range(3):
        ones = np.argwhere(si[c] == 1.0)
        lo, hi = ones.min(0), ones.max(0)
        for d in range(3):
            r = rng[d][0] if d == c else rng[d][1]
            assert lo[d] == r[0] and hi[d] == r[1] - 1
        assert np.all(si[c][si[c] != 1.0] == 1000.0)
        n_in = np.prod([(rng[d][0] if d == c else rng[d][1])[1] - (rng[d][0] if d == c else rng[d][1])[0]
                        for d in range(3)])
        assert len(ones) == n_in
    mom, ind, prm, _ = configs.full_bc(N=8, N_w=3)
    assert tuple(prm.ind_offset) == mg.sub_domain_offset(mom, ind)


def test_full_bc_case_steps_in_the_oracle():
    """The full_BC preset (mesh-bank meshes, walls, vacuum) wired into the
    oracle's step: two steps solved to 1e-12 keep div U and div B at
    round-off level and every field finite."""
    import oracle.oracle as O
    from moons_b200 import capi as G
    o = configs.make(O, configs.full_bc, seed=2, N=6, N_w=2, mqp=mg.MeshQuality(), tol=1e-12,
                     iter_max=(20000,) * 4, noise=1e-2)
    info = o.step(2)
    du, db = o.divergence()
    assert du < 1e-16 and db < 1e-22, (du, db)
    assert info["res_p"] < 1e-11
    for which in (G.MHD_U, G.MHD_B, G.MHD_J):
        for c in range(3):
            assert np.isfinite(o.download(which, c)).all()
