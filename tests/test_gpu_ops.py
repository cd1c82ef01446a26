"""GPU parity of the discrete operators and BCs against the oracle.

Each case uploads the same seeded arrays to the CUDA library (through the
C-ABI) and to the CPU oracle, runs the same reference routine on both and
compares whole arrays, ghost layers included.  FP64 stencils: the tolerance
is 1e-13 relative to the largest output entry (FMA contraction and operation
order differ between nvcc and g++)."""
import itertools

import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200.capi import (CC, FX, FY, FZ, EX, EY, EZ, NODE, DIRICHLET, NEUMANN, PERIODIC, ROBIN)
from tests.common import small_mesh_coords, rel_err, bc

pytestmark = pytest.mark.gpu
TOL = 1e-13


@pytest.fixture(scope="module")
def meshes():
    c = small_mesh_coords()
    return G.Mesh(*c), O.Mesh(*c)


def pair(meshes, dl, data=None, rng=None):
    g, o = meshes[0].field(dl), meshes[1].field(dl)
    if data is None and rng is not None:
        data = rng.standard_normal(g.shape)
    if data is not None:
        g.upload(data)
        o.upload(data)
    return g, o


def check(pg, po, tol=TOL, what=""):
    a, b = pg.download(), po.download()
    assert a.shape == b.shape
    e = rel_err(a, b)
    if not e < tol:
        bad = np.argwhere(np.abs(a - b) > tol * max(np.abs(b).max(), 1e-300))
        raise AssertionError(f"{what}: rel err {e}, {len(bad)} bad points, first {bad[:5].tolist()} shape {a.shape}")


# del for every pair of data locations that differ along dir by a flip, or are collocated
CASES = []
for dl_in in range(8):
    for d in (1, 2, 3):
        bit = 1 << (d - 1)
        from moons_b200.csrc_bits import dl_bits, dl_from_bits  # noqa
        for flip in (0, 1):
            dl_out = dl_from_bits(dl_bits(dl_in) ^ (bit if flip else 0))
            for n in ((1,) if flip else (1, 2)):
                CASES.append((dl_in, dl_out, n, d))


@pytest.mark.parametrize("dl_in,dl_out,n,d", CASES)
@pytest.mark.parametrize("pad,gen", [(0, 1), (0, 2), (0, 3), (1, 1), (1, 2)])
def test_del(meshes, dl_in, dl_out, n, d, pad, gen):
    rng = np.random.default_rng(hash((dl_in, dl_out, n, d, pad, gen)) % 2**32)
    ig, io = pair(meshes, dl_in, rng=rng)
    og, oo = pair(meshes, dl_out, rng=rng)
    G.delta(og, ig, n, d, pad, gen)
    O.delta(oo, io, n, d, pad, gen)
    check(og, oo)


def test_grad_div_curl(meshes):
    rng = np.random.default_rng(7)
    ug, uo = pair(meshes, CC, rng=rng)
    gg = [pair(meshes, d, rng=rng) for d in (FX, FY, FZ)]
    G.grad(*[p[0] for p in gg], ug)
    O.grad(*[p[1] for p in gg], uo)
    for c, p in enumerate(gg):
        check(*p, what=f"grad {c}")
    dg, do = pair(meshes, CC, rng=rng)
    G.div(dg, *[p[0] for p in gg])
    O.div(do, *[p[1] for p in gg])
    check(dg, do, what="div")
    # curl of random faces (curl of the gradient above is zero up to rounding)
    rf = [pair(meshes, d, rng=rng) for d in (FX, FY, FZ)]
    eg = [pair(meshes, d, rng=rng) for d in (EX, EY, EZ)]
    G.curl([p[0] for p in eg], [p[0] for p in rf])
    O.curl([p[1] for p in eg], [p[1] for p in rf])
    for c, p in enumerate(eg):
        check(*p, what=f"curl F->E {c}")
    fg = [pair(meshes, d, rng=rng) for d in (FX, FY, FZ)]
    G.curl([p[0] for p in fg], [p[0] for p in eg])
    O.curl([p[1] for p in fg], [p[1] for p in eg])
    for c, p in enumerate(fg):
        check(*p, what=f"curl E->F {c}")


@pytest.mark.parametrize("dl", [CC, FX, FY, FZ, EX, EY, EZ, NODE])
def test_lap_centered(meshes, dl):
    rng = np.random.default_rng(11 + dl)
    ug, uo = pair(meshes, dl, rng=rng)
    og, oo = pair(meshes, dl, rng=rng)
    G.lap_centered(og, ug)
    O.lap_centered(oo, uo)
    check(og, oo)


def test_lap_var(meshes):
    rng = np.random.default_rng(5)
    ug, uo = pair(meshes, CC, rng=rng)
    ks = [pair(meshes, d, data=np.exp(rng.standard_normal(meshes[0].field(d).shape))) for d in (FX, FY, FZ)]
    og, oo = pair(meshes, CC, rng=rng)
    G.lap_var(og, ug, [k[0] for k in ks])
    O.lap_var(oo, uo, [k[1] for k in ks])
    check(og, oo)


@pytest.mark.parametrize("dl_in,d", [(dl, d) for dl in range(8) for d in (1, 2, 3)])
def test_interp(meshes, dl_in, d):
    from moons_b200.csrc_bits import dl_bits, dl_from_bits
    rng = np.random.default_rng(dl_in * 3 + d)
    dl_out = dl_from_bits(dl_bits(dl_in) ^ (1 << (d - 1)))
    ig, io = pair(meshes, dl_in, rng=rng)
    og, oo = pair(meshes, dl_out, rng=rng)
    G.interp(og, ig, d)
    O.interp(oo, io, d)
    check(og, oo)


BC_SETS = [
    [DIRICHLET] * 6,
    [NEUMANN] * 6,
    [PERIODIC, PERIODIC, NEUMANN, DIRICHLET, NEUMANN, NEUMANN],
    [DIRICHLET, NEUMANN, PERIODIC, PERIODIC, ROBIN, ROBIN],
    [ROBIN, ROBIN, DIRICHLET, DIRICHLET, PERIODIC, PERIODIC],
]


@pytest.mark.parametrize("types", BC_SETS)
@pytest.mark.parametrize("dl", [CC, FX, FY, FZ, EX, EY, EZ])
@pytest.mark.parametrize("implicit", [False, True])
@pytest.mark.parametrize("prescribed", [0, 1])
def test_bcs(meshes, types, dl, implicit, prescribed):
    rng = np.random.default_rng(hash((tuple(types), dl, implicit, prescribed)) % 2**32)
    spec = bc(types, values=rng.standard_normal(6), c_w=[0.5 + i for i in range(6)],
              prescribed=[prescribed] * 6, order=[5, 6, 1, 2, 3, 4])
    ug, uo = pair(meshes, dl, rng=rng)
    ug.set_bcs(spec)
    uo.set_bcs(spec)
    if implicit:
        ug.apply_bcs_implicit()
        uo.apply_bcs_implicit()
    else:
        ug.apply_bcs()
        uo.apply_bcs()
    check(ug, uo, 1e-15)
