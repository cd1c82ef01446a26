"""Multigrid-preconditioned CG (FP64 V-cycle) and its mixed-precision form
(FP32 V-cycle in FP64 flexible CG) against the oracle's Jacobi-PCG on the
same systems: both must reach the tolerance and agree on the solution (up to
the constant of all-Neumann problems)."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200.capi import CC, FX, FY, FZ, NEUMANN, DIRICHLET, PERIODIC, OP_LAP_UNIFORM, OP_LAP_PROPS, PREC_LAP, isp
from tests.common import coords, bc

pytestmark = pytest.mark.gpu


def mesh_coords(n, stretched):
    kinds = ("roberts", "uniform", "roberts") if stretched else ("uniform",) * 3
    return [coords(k, nn, 0.0, 1.0 + 0.5 * i, 1.05 + 0.1 * i) for i, (k, nn) in enumerate(zip(kinds, n))]


def interior(a):
    return a[1:-1, 1:-1, 1:-1]


def solve_pair(n, bctypes, alln, prec, stretched=True, props=False, seed=0):
    cs = mesh_coords(n, stretched)
    mg_, mo = G.Mesh(*cs), O.Mesh(*cs)
    rng = np.random.default_rng(seed)
    pg, po = mg_.field(CC), mo.field(CC)
    spec = bc(bctypes, all_neumann=alln)
    pg.set_bcs(spec)
    po.set_bcs(spec)
    s = pg.shape
    bg, bo = mg_.field(CC), mo.field(CC)
    b = rng.standard_normal(s)
    bg.upload(b)
    bo.upload(b)
    kg = ko = None
    if props:
        kg, ko = [], []
        for ax, d in enumerate((FX, FY, FZ)):
            a, c = mg_.field(d), mo.field(d)
            v = 10.0 ** rng.uniform(-1, 1, a.shape)
            if bctypes[2 * ax] == PERIODIC:
                # one physical face at the periodic seam: the same coefficient on both copies
                sl_lo = [slice(None)] * 3
                sl_hi = [slice(None)] * 3
                sl_lo[ax] = 1
                sl_hi[ax] = v.shape[ax] - 2
                v[tuple(sl_hi)] = v[tuple(sl_lo)]
            a.upload(v)
            c.upload(v)
            kg.append(a)
            ko.append(c)
    op = OP_LAP_PROPS if props else OP_LAP_UNIFORM
    sg = G.PCG(mg_, op, prec, [pg], [pg], kg)
    so = O.PCG(mo, op, PREC_LAP, [po], [po], ko)
    par = isp(5000, 1e-10, 1e-300)
    ig = sg.solve([pg], [bg], par)
    io = so.solve([po], [bo], par)
    return ig, io, pg.download(), po.download(), alln


CASES = [
    ((16, 16, 16), [NEUMANN] * 6, True),
    ((16, 8, 32), [NEUMANN, NEUMANN, NEUMANN, NEUMANN, PERIODIC, PERIODIC], True),
    ((16, 16, 8), [DIRICHLET, DIRICHLET, NEUMANN, NEUMANN, NEUMANN, DIRICHLET], False),
    ((8, 16, 16), [PERIODIC, PERIODIC, DIRICHLET, NEUMANN, PERIODIC, PERIODIC], False),
    # odd cell counts: pairs plus one unpaired cell per coarsening
    ((15, 9, 13), [NEUMANN] * 6, True),
    ((13, 8, 21), [NEUMANN, NEUMANN, NEUMANN, NEUMANN, PERIODIC, PERIODIC], True),
    ((9, 17, 7), [DIRICHLET, DIRICHLET, NEUMANN, NEUMANN, NEUMANN, DIRICHLET], False),
    ((12, 17, 10), [PERIODIC, PERIODIC, DIRICHLET, NEUMANN, PERIODIC, PERIODIC], False),
]


@pytest.mark.parametrize("prec", [G.PREC_MG, G.PREC_MG_MIXED])
@pytest.mark.parametrize("n,bctypes,alln", CASES)
@pytest.mark.parametrize("props", [False, True])
def test_mgpcg_matches_jacobi_pcg(n, bctypes, alln, prec, props):
    ig, io, xg, xo, alln = solve_pair(n, bctypes, alln, prec, props=props)
    assert ig["exit_reason"] == 1 and io["exit_reason"] == 1, (ig, io)
    assert ig["rel"] < 1e-10
    assert abs(ig["res0"] - io["res0"]) <= 1e-12 * io["res0"]
    # far fewer iterations than Jacobi
    assert ig["iterations"] <= 0.5 * io["iterations"], (ig, io)
    a, b = interior(xg), interior(xo)
    if alln:
        a = a - a.mean()
        b = b - b.mean()
    err = np.abs(a - b).max() / np.abs(b).max()
    assert err < 1e-7, err


@pytest.mark.parametrize("n,bctypes,alln", CASES)
def test_fast_diagonalization_is_a_direct_solve(n, bctypes, alln):
    """MOONS_PREC_FD: the separable operator's exact inverse as the
    preconditioner; CG stops after one or two iterations at the tolerance
    with the Jacobi-PCG solution."""
    ig, io, xg, xo, alln = solve_pair(n, bctypes, alln, G.PREC_FD)
    assert ig["exit_reason"] == 1 and io["exit_reason"] == 1, (ig, io)
    assert ig["rel"] < 1e-10
    assert abs(ig["res0"] - io["res0"]) <= 1e-12 * io["res0"]
    assert ig["iterations"] <= 3, ig
    a, b = interior(xg), interior(xo)
    if alln:
        a = a - a.mean()
        b = b - b.mean()
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-7


def test_fast_diagonalization_needs_a_separable_operator():
    with pytest.raises(G.MoonsError):
        solve_pair((8, 8, 8), [NEUMANN] * 6, True, G.PREC_FD, props=True)
