"""CPU checks of the multigrid restatement (oracle/mg_oracle.py) against the
C++ oracle and its own algebra: the level residual equals vol * the oracle's
lap_centered with implicit BCs; the restriction is the transpose of the
prolongation; prolongation reproduces linear functions along a coarsened
uniform axis away from the boundary; the red-black sweeps reduce the
residual; restrict_c keeps every other node of an even axis."""
import numpy as np
import pytest

import oracle.mg_oracle as MO
import oracle.oracle as O
from moons_b200 import capi as G
from tests.common import coords

BCT = [1, 2, 2, 1, 1, 2]


def meshes():
    return [coords(k, n, 0.0, 1.0 + 0.3 * i, 1.05 + 0.1 * i)
            for i, (k, n) in enumerate(zip(("roberts", "roberts", "uniform"), (14, 9, 11)))]


def test_residual_is_the_oracle_operator():
    hs = meshes()
    shp = tuple(len(h) - 1 for h in hs)
    rng = np.random.default_rng(0)
    I = (slice(1, -1),) * 3
    r = np.zeros(shp)
    e = np.zeros(shp)
    r[I] = rng.standard_normal(tuple(x - 2 for x in shp))
    e[I] = rng.standard_normal(tuple(x - 2 for x in shp))
    m = O.Mesh(*hs)
    f = m.field(G.CC)
    f.set_bcs(G.bc_spec(BCT))
    f.upload(e)
    f.apply_bcs_implicit()
    lf = m.field(G.CC)
    O.lap_centered(lf, f)
    want = r - MO.vol(hs) * lf.download()
    got = MO.residual(e, r, hs, BCT)
    assert np.abs(got[I] - want[I]).max() < 1e-14 * np.abs(want[I]).max()


def test_restriction_is_the_transpose():
    hs = meshes()
    hc = [MO.coarse_nodes(h) for h in hs]
    s0 = tuple(len(h) - 1 for h in hs)
    s1 = tuple(len(h) - 1 for h in hc)
    rng = np.random.default_rng(1)
    I = (slice(1, -1),) * 3
    ec = np.zeros(s1)
    tf = np.zeros(s0)
    ec[I] = rng.standard_normal(tuple(x - 2 for x in s1))
    tf[I] = rng.standard_normal(tuple(x - 2 for x in s0))
    a = np.sum(MO.prolong(ec, hc, s0, BCT)[I] * tf[I])
    b = np.sum(ec[I] * MO.restrict(tf, hc, s1, BCT)[I])
    assert abs(a - b) < 1e-13 * abs(a)


def test_prolongation_is_linear_interpolation_inside():
    h = np.linspace(0.0, 1.0, 17)
    hn = MO.add_ghost_nodes(h)
    hc = MO.coarse_nodes(hn)
    xc = 0.5 * (hc[1:] + hc[:-1])
    xf = 0.5 * (hn[1:] + hn[:-1])
    u = np.tile((2.0 + 3.0 * xc)[:, None, None], (1, 3, 3))
    p = MO.prolong_axis(u, hc, 0, 16, MO.NEUMANN, MO.NEUMANN)
    inner = slice(2, -2)
    # each fine cell: mean of its parent and the face value -> the value at
    # the point midway between them (exact for a linear function)
    want = 2.0 + 3.0 * xf
    assert np.abs(p[inner, 1, 1] - want[inner]).max() < 1e-12


def test_sweeps_reduce_the_residual():
    hs = meshes()
    shp = tuple(len(h) - 1 for h in hs)
    rng = np.random.default_rng(2)
    I = (slice(1, -1),) * 3
    r = np.zeros(shp)
    r[I] = rng.standard_normal(tuple(x - 2 for x in shp))
    e = np.zeros(shp)
    n0 = np.linalg.norm(MO.residual(e, r, hs, BCT))
    for _ in range(10):
        e = MO.red_black(e, r, hs, BCT, 1.15)
    assert np.linalg.norm(MO.residual(e, r, hs, BCT)) < 0.2 * n0


@pytest.mark.parametrize("n", [8, 16])
def test_restrict_c_keeps_every_other_node(n):
    h = np.sort(np.random.default_rng(n).uniform(0, 1, n + 1))
    hn = MO.add_ghost_nodes(h)
    hc = MO.coarse_nodes(hn)
    assert np.array_equal(hc[1:-1], h[0::2])
