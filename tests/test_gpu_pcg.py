"""GPU parity of the PCG solver object (PCG_solver_SF/VF) against the oracle.

Both sides run the reference algorithm with the same exit tests, so the
iteration counts agree (+-1 where the last residual sits at the tolerance)
and the solutions agree to well below the solver tolerance."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200.capi import (CC, FX, FY, FZ, EX, EY, EZ, DIRICHLET, NEUMANN, PERIODIC, ROBIN, OP_LAP_UNIFORM,
                             OP_LAP_PROPS, OP_MOM_DIFFUSION, OP_IND_DIFFUSION, OP_NRG_DIFFUSION, PREC_LAP, PREC_MOM,
                             PREC_IND,
                             PREC_IDENTITY, isp)
from tests.common import small_mesh_coords, rel_err, bc

pytestmark = pytest.mark.gpu


def both(coords):
    return G.Mesh(*coords), O.Mesh(*coords)


def fields(ms, dls, data):
    out = []
    for dl, a in zip(dls, data):
        g, o = ms[0].field(dl), ms[1].field(dl)
        if a is not None:
            g.upload(a)
            o.upload(a)
        out.append((g, o))
    return out


def run_both(ms, op, prec, xs, xbcs, bs, params, ks=None, coeff=None):
    sg = G.PCG(ms[0], op, prec, [x[0] for x in xs], [x[0] for x in xbcs], [k[0] for k in ks] if ks else None)
    so = O.PCG(ms[1], op, prec, [x[1] for x in xs], [x[1] for x in xbcs], [k[1] for k in ks] if ks else None)
    if coeff is not None:
        sg.update_mfp(coeff, True)
        so.update_mfp(coeff, True)
    ig = sg.solve([x[0] for x in xs], [b[0] for b in bs], params)
    io = so.solve([x[1] for x in xs], [b[1] for b in bs], params)
    return ig, io


def shape(m, dl):
    return m.field(dl).shape


@pytest.mark.parametrize("bctypes,alln", [([NEUMANN] * 6, True),
                                          ([PERIODIC, PERIODIC, NEUMANN, NEUMANN, NEUMANN, NEUMANN], True),
                                          ([DIRICHLET] * 6, False)])
@pytest.mark.parametrize("stretched", [False, True])
def test_pcg_lap_uniform_sf(bctypes, alln, stretched):
    ms = both(small_mesh_coords(stretched=stretched))
    rng = np.random.default_rng(1)
    s = shape(ms[1], CC)
    (p,) = fields(ms, [CC], [np.zeros(s)])
    spec = bc(bctypes, all_neumann=alln, order=[5, 6, 1, 2, 3, 4])
    p[0].set_bcs(spec)
    p[1].set_bcs(spec)
    (b,) = fields(ms, [CC], [rng.standard_normal(s)])
    ig, io = run_both(ms, OP_LAP_UNIFORM, PREC_LAP, [p], [p], [b], isp(3000, 1e-10, 1e-15))
    assert ig["exit_reason"] == io["exit_reason"]
    assert abs(ig["iterations"] - io["iterations"]) <= 1, (ig, io)
    assert abs(ig["res0"] - io["res0"]) <= 1e-12 * io["res0"]
    assert rel_err(p[0].download(), p[1].download()) < 1e-9


def test_pcg_fixed_iterations_match_exactly():
    # with a fixed iteration budget both sides run the same recurrence
    ms = both(small_mesh_coords())
    rng = np.random.default_rng(2)
    s = shape(ms[1], CC)
    (p,) = fields(ms, [CC], [rng.standard_normal(s)])
    spec = bc([NEUMANN] * 6, all_neumann=True)
    p[0].set_bcs(spec)
    p[1].set_bcs(spec)
    (b,) = fields(ms, [CC], [rng.standard_normal(s)])
    ig, io = run_both(ms, OP_LAP_UNIFORM, PREC_LAP, [p], [p], [b], isp(25, 0.0, 0.0))
    assert ig["iterations"] == io["iterations"] == 25
    assert abs(ig["res"] - io["res"]) < 1e-10 * io["res"]
    assert rel_err(p[0].download(), p[1].download()) < 1e-11


def test_pcg_lap_props_sigma():
    ms = both(small_mesh_coords())
    rng = np.random.default_rng(3)
    s = shape(ms[1], CC)
    (phi,) = fields(ms, [CC], [np.zeros(s)])
    spec = bc([DIRICHLET, DIRICHLET, NEUMANN, NEUMANN, NEUMANN, NEUMANN])
    phi[0].set_bcs(spec)
    phi[1].set_bcs(spec)
    ks = fields(ms, [FX, FY, FZ], [10.0 ** rng.uniform(-3, 3, shape(ms[1], d)) for d in (FX, FY, FZ)])
    (b,) = fields(ms, [CC], [rng.standard_normal(s)])
    ig, io = run_both(ms, OP_LAP_PROPS, PREC_LAP, [phi], [phi], [b], isp(5000, 1e-10, 1e-15), ks=ks)
    # six decades of coefficient contrast: thousands of iterations, whose count
    # moves by a few tens with the order of the floating-point sums (CG loses
    # orthogonality at this conditioning); both runs must reach the tolerance
    assert abs(ig["iterations"] - io["iterations"]) <= max(1, 0.02 * io["iterations"]), (ig, io)
    assert ig["rel"] < 1e-10 and io["rel"] < 1e-10
    assert rel_err(phi[0].download(), phi[1].download()) < 1e-7


@pytest.mark.parametrize("bctypes", [[DIRICHLET, DIRICHLET, NEUMANN, NEUMANN, DIRICHLET, NEUMANN],
                                     [NEUMANN, NEUMANN, DIRICHLET, DIRICHLET, PERIODIC, PERIODIC]])
def test_pcg_nrg_diffusion(bctypes):
    """The energy equation's implicit operator I + c div(k grad) with the
    reference's prec_lap_SF (energy_extend.f90:129), T at cell centres."""
    ms = both(small_mesh_coords())
    rng = np.random.default_rng(9)
    s = shape(ms[1], CC)
    (T,) = fields(ms, [CC], [rng.standard_normal(s) * 0.1])
    spec = bc(bctypes, values=[1.0, 0.0, 0.0, 0.0, 0.5, 0.0])
    T[0].set_bcs(spec)
    T[1].set_bcs(spec)
    ks = fields(ms, [FX, FY, FZ], [10.0 ** rng.uniform(-1, 1, shape(ms[1], d)) for d in (FX, FY, FZ)])
    (b,) = fields(ms, [CC], [rng.standard_normal(s)])
    ig, io = run_both(ms, OP_NRG_DIFFUSION, PREC_LAP, [T], [T], [b], isp(3000, 1e-10, 1e-15), ks=ks, coeff=-0.02)
    assert ig["exit_reason"] == io["exit_reason"] == 1
    assert abs(ig["iterations"] - io["iterations"]) <= 1, (ig, io)
    assert rel_err(T[0].download(), T[1].download()) < 1e-9


def test_pcg_mom_diffusion_vf():
    ms = both(small_mesh_coords())
    rng = np.random.default_rng(4)
    dls = [FX, FY, FZ]
    U = fields(ms, dls, [rng.standard_normal(shape(ms[1], d)) * 0.1 for d in dls])
    for c, (g, o) in enumerate(U):
        vals = [0.0] * 6
        if c == 0:
            vals[3] = 1.0  # lid (LDC_at_ymax)
        spec = bc([DIRICHLET] * 6, values=vals, order=[5, 6, 1, 2, 3, 4])
        g.set_bcs(spec)
        o.set_bcs(spec)
    B = fields(ms, dls, [rng.standard_normal(shape(ms[1], d)) for d in dls])
    ig, io = run_both(ms, OP_MOM_DIFFUSION, PREC_MOM, U, U, B, isp(500, 1e-10, 1e-15), coeff=-1e-3 / 400.0 * 50)
    assert abs(ig["iterations"] - io["iterations"]) <= 1, (ig, io)
    for g, o in U:
        assert rel_err(g.download(), o.download()) < 1e-9


DUCT_B = [[NEUMANN, NEUMANN, DIRICHLET, DIRICHLET, PERIODIC, PERIODIC],
          [DIRICHLET, DIRICHLET, NEUMANN, NEUMANN, PERIODIC, PERIODIC],
          [DIRICHLET, DIRICHLET, DIRICHLET, DIRICHLET, PERIODIC, PERIODIC]]


@pytest.mark.parametrize("op", ["mom", "ind"])
def test_pcg_vf_duct_bcs(op):
    # per-component BC patterns of the duct (pseudo-vacuum B, periodic streamwise)
    ms = both(small_mesh_coords())
    rng = np.random.default_rng(9)
    dls = [FX, FY, FZ]
    X = fields(ms, dls, [np.zeros(shape(ms[1], d)) for d in dls])
    for c, (g, o) in enumerate(X):
        types = DUCT_B[c] if op == "ind" else [DIRICHLET] * 4 + [PERIODIC] * 2
        spec = bc(types, prescribed=[0, 0, 0, 0, 1, 1])
        g.set_bcs(spec)
        o.set_bcs(spec)
    R = fields(ms, dls, [rng.standard_normal(shape(ms[1], d)) for d in dls])
    if op == "ind":
        sig = fields(ms, [EX, EY, EZ], [1.0 / (10.0 ** rng.uniform(-1, 1, shape(ms[1], d))) for d in (EX, EY, EZ)])
        ig, io = run_both(ms, OP_IND_DIFFUSION, PREC_IND, X, X, R, isp(800, 1e-12, 1e-15), ks=sig, coeff=0.05)
    else:
        ig, io = run_both(ms, OP_MOM_DIFFUSION, PREC_MOM, X, X, R, isp(800, 1e-12, 1e-15), coeff=-0.05)
    assert abs(ig["iterations"] - io["iterations"]) <= 1, (ig, io)
    for g, o in X:
        assert rel_err(g.download(), o.download()) < 1e-8


def test_pcg_ind_diffusion_vf():
    ms = both(small_mesh_coords())
    rng = np.random.default_rng(5)
    dls = [FX, FY, FZ]
    Bf = fields(ms, dls, [np.zeros(shape(ms[1], d)) for d in dls])
    for c, (g, o) in enumerate(Bf):
        types = [DIRICHLET] * 6
        types[2 * c] = NEUMANN
        types[2 * c + 1] = NEUMANN  # pseudo_vacuum (init_B_BCs.f90:83-97)
        spec = bc(types)
        g.set_bcs(spec)
        o.set_bcs(spec)
    sig = fields(ms, [EX, EY, EZ], [1.0 / (10.0 ** rng.uniform(-1, 1, shape(ms[1], d))) for d in (EX, EY, EZ)])
    R = fields(ms, dls, [rng.standard_normal(shape(ms[1], d)) for d in dls])
    ig, io = run_both(ms, OP_IND_DIFFUSION, PREC_IND, Bf, Bf, R, isp(800, 1e-10, 1e-15), ks=sig, coeff=0.05)
    assert abs(ig["iterations"] - io["iterations"]) <= 1, (ig, io)
    for g, o in Bf:
        assert rel_err(g.download(), o.download()) < 1e-8
