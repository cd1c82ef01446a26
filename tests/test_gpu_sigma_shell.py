"""The mixed-precision Poisson case (sigma-weighted Laplacian with a
high-contrast wall shell, RHS = div(u x B)) on a small grid: the multigrid
(FP64 and FP32 V-cycle) solves reach the tolerance and agree with the
oracle's Jacobi-PCG solution."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200 import configs
from moons_b200.capi import CC, FX, FY, FZ, NEUMANN, OP_LAP_PROPS, PREC_LAP, isp
from tests.common import bc

pytestmark = pytest.mark.gpu


def build(backend, n, shell, seed):
    coords, sig, E = configs.sigma_shell(n, shell, seed)
    m = backend.Mesh(*coords)
    phi = m.field(CC)
    phi.set_bcs(bc([NEUMANN] * 6, all_neumann=True))
    ks, es = [], []
    for d, dl in enumerate((FX, FY, FZ)):
        k = m.field(dl)
        k.upload(sig[d])
        ks.append(k)
        e = m.field(dl)
        e.upload(E[d])
        es.append(e)
    rhs = m.field(CC)
    backend.div(rhs, *es)
    return m, phi, ks, rhs


@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("prec", [G.PREC_MG, G.PREC_MG_MIXED], ids=["mg", "mixed"])
def test_sigma_shell_multigrid_matches_oracle(prec, seed):
    n, shell = 16, 2
    mg_, pg, kg, bg = build(G, n, shell, seed)
    mo, po, ko, bo = build(O, n, shell, seed)
    assert np.abs(bg.download() - bo.download()).max() <= 1e-12 * np.abs(bo.download()).max()
    sg = G.PCG(mg_, OP_LAP_PROPS, prec, [pg], [pg], kg)
    so = O.PCG(mo, OP_LAP_PROPS, PREC_LAP, [po], [po], ko)
    par = isp(20000, 1e-10, 1e-300)
    ig = sg.solve([pg], [bg], par)
    io = so.solve([po], [bo], par)
    assert ig["exit_reason"] == 1 and io["exit_reason"] == 1, (ig, io)
    assert ig["iterations"] < io["iterations"], (ig, io)
    a = pg.download()[1:-1, 1:-1, 1:-1]
    b = po.download()[1:-1, 1:-1, 1:-1]
    a = a - a.mean()
    b = b - b.mean()
    assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()
