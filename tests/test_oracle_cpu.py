"""CPU checks of the oracle against the reference's own verification
routines (identities, Poisson residual drop, SPD symmetry)."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200.capi import (CC, FX, FY, FZ, EX, EY, EZ, NEUMANN, DIRICHLET, PERIODIC, OP_LAP_UNIFORM, PREC_LAP,
                             OP_MOM_DIFFUSION, PREC_MOM, isp)
from tests.common import small_mesh_coords, bc


@pytest.fixture(scope="module")
def mesh():
    return O.Mesh(*small_mesh_coords())


def test_curl_grad_zero(mesh):
    # operator_commute_test.f90:52-80: curl(grad phi) = 0 on random phi
    rng = np.random.default_rng(1)
    u = mesh.field(CC)
    u.upload(rng.standard_normal(u.shape))
    g = [mesh.field(d) for d in (FX, FY, FZ)]
    O.grad(*g, u)
    c = [mesh.field(d) for d in (EX, EY, EZ)]
    O.curl(c, g)
    scale = max(np.abs(x.download()).max() for x in g)
    err = max(np.abs(x.download()[1:-1, 1:-1, 1:-1]).max() for x in c)
    assert err < 1e-12 * scale * 100


def test_div_curl_zero(mesh):
    rng = np.random.default_rng(2)
    e = [mesh.field(d) for d in (EX, EY, EZ)]
    for x in e:
        x.upload(rng.standard_normal(x.shape))
    f = [mesh.field(d) for d in (FX, FY, FZ)]
    O.curl(f, e)
    dv = mesh.field(CC)
    O.div(dv, *f)
    scale = max(np.abs(x.download()).max() for x in f)
    assert np.abs(dv.download()[1:-1, 1:-1, 1:-1]).max() < 1e-12 * scale * 100


def test_poisson_residual_drop(mesh):
    # Poisson_test.f90:50-93: all-Neumann CC Poisson, random source
    rng = np.random.default_rng(3)
    p = mesh.field(CC)
    p.set_bcs(bc([NEUMANN] * 6, all_neumann=True))
    b = mesh.field(CC)
    b.upload(rng.standard_normal(b.shape))
    s = O.PCG(mesh, OP_LAP_UNIFORM, PREC_LAP, [p], [p])
    info = s.solve([p], [b], isp(2000, 1e-10, 1e-16))
    assert info["exit_reason"] == 1 and info["rel"] < 1e-10


def test_laplacian_symmetry_vol_weighted():
    # test_symmetry_SF (HW/sparse/matrix.f90:53-89): <vol A x, y> = <x, vol A y>
    m = O.Mesh(*small_mesh_coords(n=(6, 5, 4)))
    rng = np.random.default_rng(4)
    x, y = m.field(CC), m.field(CC)
    spec = bc([NEUMANN] * 6)
    x.set_bcs(spec)
    y.set_bcs(spec)
    xa = np.zeros(x.shape)
    ya = np.zeros(x.shape)
    xa[1:-1, 1:-1, 1:-1] = rng.standard_normal((x.shape[0] - 2, x.shape[1] - 2, x.shape[2] - 2))
    ya[1:-1, 1:-1, 1:-1] = rng.standard_normal((x.shape[0] - 2, x.shape[1] - 2, x.shape[2] - 2))
    x.upload(xa)
    y.upload(ya)
    x.apply_bcs_implicit()
    y.apply_bcs_implicit()
    ax, ay = m.field(CC), m.field(CC)
    O.lap_centered(ax, x)
    O.lap_centered(ay, y)
    hx, hy, hz = [np.diff(h) for h in m._keep]
    vol = np.einsum("i,j,k->ijk", hx, hy, hz)
    I = (slice(1, -1),) * 3
    lhs = np.sum((vol * ax.download())[I] * ya[I])
    rhs = np.sum(xa[I] * (vol * ay.download())[I])
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)
