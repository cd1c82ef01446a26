"""The multigrid building blocks one at a time, through the diagnostic C-ABI
entry (moons_mg_debug), against the CPU restatement in oracle/mg_oracle.py:

* the coarse level's node coordinates (restrict_c, coordinates_extend.f90:336-356,
  with the library's extensions for odd counts and periodic ghosts);
* prolongation = prolongate_C (GF_prolongate.f90:22-56) per coarsened axis;
* restriction = its transpose (checked directly and by <P a, t> = <a, R t>);
* one red and one black SOR sweep = the redBlack point update
  (SOR.f90:234-268) on the red / black parity patterns, the homogeneous
  ghost image of a boundary point taken into the divisor;
* the level residual r - A e.
Meshes: Roberts-stretched and uniform axes, even and odd cell counts,
Dirichlet / Neumann / periodic faces.  Bound: 1e-13 relative (one pass of
each operator; the sums are added in different orders)."""
import numpy as np
import pytest

import oracle.mg_oracle as MO
from moons_b200 import capi as G
from tests.common import coords

pytestmark = pytest.mark.gpu

D, N, P = G.DIRICHLET, G.NEUMANN, G.PERIODIC

CASES = {
    "neumann_even_stretched": ((16, 12, 10), ("roberts", "uniform", "roberts"), [N] * 6, True),
    "mixed_odd": ((14, 9, 11), ("roberts", "roberts", "uniform"), [D, N, N, D, D, N], False),
    "periodic_x": ((16, 10, 12), ("uniform", "roberts", "roberts"), [P, P, N, D, N, N], False),
}


def setup(name):
    n, kinds, bct, alln = CASES[name]
    hs = [coords(k, nn, 0.0, 1.0 + 0.3 * i, 1.05 + 0.1 * i) for i, (k, nn) in enumerate(zip(kinds, n))]
    m = G.Mesh(*hs)
    x = m.field(G.CC)
    x.set_bcs(G.bc_spec(bct, all_neumann=alln))
    s = G.PCG(m, G.OP_LAP_UNIFORM, G.PREC_MG, [x], [x])
    return s, hs, bct


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def levels(s, hs, bct):
    (s0, _), nl = s.mg_level_shape(0), s.mg_level_shape(0)[1]
    assert nl >= 2
    shp0 = s.mg_level_shape(0)[0]
    shp1 = s.mg_level_shape(1)[0]
    assert shp0 == tuple(len(h) - 1 for h in hs)
    hc = []
    for d in range(3):
        if shp1[d] == shp0[d]:
            hc.append(np.asarray(hs[d]))
        else:
            hc.append(MO.coarse_nodes(hs[d], periodic=bct[2 * d] == P))
        assert len(hc[d]) - 1 == shp1[d], (d, len(hc[d]), shp1)
    return shp0, shp1, hc


@pytest.mark.parametrize("name", list(CASES))
def test_prolongation_and_restriction(name):
    s, hs, bct = setup(name)
    shp0, shp1, hc = levels(s, hs, bct)
    rng = np.random.default_rng(4)
    ec = np.zeros(shp1)
    ec[1:-1, 1:-1, 1:-1] = rng.standard_normal(tuple(x - 2 for x in shp1))
    got = s.mg_debug(0, 0, ec)
    want = MO.prolong(ec, hc, shp0, bct)
    I = (slice(1, -1),) * 3
    assert rel(got[I], want[I]) < 1e-13
    tf = np.zeros(shp0)
    tf[I] = rng.standard_normal(tuple(x - 2 for x in shp0))
    gr = s.mg_debug(1, 0, tf)
    wr = MO.restrict(tf, hc, shp1, bct)
    assert rel(gr, wr) < 1e-13
    # adjointness of the library's own pair
    assert abs(np.sum(got[I] * tf[I]) - np.sum(ec[I] * gr[I])) < 1e-12 * abs(np.sum(got[I] * tf[I]))


@pytest.mark.parametrize("name", list(CASES))
def test_red_black_sweep_and_residual(name):
    s, hs, bct = setup(name)
    shp0, _, _ = levels(s, hs, bct)
    rng = np.random.default_rng(5)
    I = (slice(1, -1),) * 3
    e = np.zeros(shp0)
    r = np.zeros(shp0)
    e[I] = rng.standard_normal(tuple(x - 2 for x in shp0))
    r[I] = rng.standard_normal(tuple(x - 2 for x in shp0))
    got = s.mg_debug(2, 0, e, r)
    want = MO.red_black(e, r, hs, bct, 1.15)
    assert rel(got[I], want[I]) < 1e-13
    t = s.mg_debug(3, 0, e, r)
    tw = MO.residual(e, r, hs, bct)
    assert rel(t[I], tw[I]) < 1e-13


def test_sweeps_reduce_the_residual():
    s, hs, bct = setup("mixed_odd")
    shp0, _, _ = levels(s, hs, bct)
    rng = np.random.default_rng(6)
    I = (slice(1, -1),) * 3
    r = np.zeros(shp0)
    r[I] = rng.standard_normal(tuple(x - 2 for x in shp0))
    e = np.zeros(shp0)
    n0 = np.linalg.norm(s.mg_debug(3, 0, e, r))
    for _ in range(20):
        e = s.mg_debug(2, 0, e, r)
    assert np.linalg.norm(s.mg_debug(3, 0, e, r)) < 0.5 * n0
