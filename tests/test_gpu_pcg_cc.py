"""GPU parity of the cell-centred PCG path against the oracle: the operator
step that stages p through shared memory and forms the ghost values from the
interior (no BC fill), with Minv formed per point.

Every CC BC kind on every face (Dirichlet, Neumann, periodic on each axis,
Robin, no BC defined), meshes whose interior does not fill the 32 x 8 tiles
(odd extents, so that staged rows start on odd elements), and single-plane
chunks; LAP_UNIFORM, LAP_PROPS and NRG_DIFFUSION.  With a fixed iteration
budget both sides run the same recurrence, so the iterates agree to
round-off; to tolerance (SPD cases) the iteration counts agree within one."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200.capi import (CC, FX, FY, FZ, DIRICHLET, NEUMANN, PERIODIC, ROBIN, OP_LAP_UNIFORM, OP_LAP_PROPS,
                             OP_NRG_DIFFUSION, PREC_LAP, isp)
from tests.common import coords, rel_err, bc

pytestmark = pytest.mark.gpu

D, N, P, R = DIRICHLET, NEUMANN, PERIODIC, ROBIN

MESHES = {
    "small": (12, 10, 8),
    "partial_tiles_odd": (37, 21, 45),   # s0 = 39 (odd): row copies start on odd elements
    "wide_thin": (70, 9, 5),
    "tall": (5, 33, 64),
}

BCSETS = {
    "neumann": ([N] * 6, True),
    "dirichlet": ([D] * 6, False),
    "periodic_x": ([P, P, N, N, N, N], True),
    "periodic_y": ([D, N, P, P, N, D], False),
    "periodic_z": ([N, D, N, N, P, P], False),
    "periodic_all": ([P] * 6, True),
    "robin": ([R, R, N, D, R, N], False),
    "undefined": (None, False),
}


def meshes(name, stretched=True):
    n = MESHES[name]
    kinds = ("roberts", "uniform", "roberts") if stretched else ("uniform",) * 3
    cs = [coords(k, nn, 0.0, 1.0 + 0.4 * i, 1.05 + 0.1 * i) for i, (k, nn) in enumerate(zip(kinds, n))]
    return G.Mesh(*cs), O.Mesh(*cs)


def setup(ms, bcset, seed, x0=True, values=(0.1, -0.2, 0.0, 0.3, 0.0, 0.05)):
    rng = np.random.default_rng(seed)
    types, alln = BCSETS[bcset]
    out = []
    s = ms[1].field(CC).shape
    xa = rng.standard_normal(s) if x0 else np.zeros(s)
    ba = rng.standard_normal(s)
    for m in ms:
        x, b = m.field(CC), m.field(CC)
        x.upload(xa)
        b.upload(ba)
        if types is not None:
            x.set_bcs(bc(types, c_w=[0.3, 0.7, 1.0, 1.0, 0.5, 1.0], values=list(values),
                         all_neumann=alln, order=[5, 6, 1, 2, 3, 4]))
        out.append((x, b))
    return out


def solve_both(ms, op, fb, params, ks=None, coeff=None):
    res = []
    for side, (m, M) in enumerate(zip(ms, (G, O))):
        x, b = fb[side]
        k = [kk[side] for kk in ks] if ks else None
        s = M.PCG(m, op, PREC_LAP, [x], [x], k)
        if coeff is not None:
            s.update_mfp(coeff, True)
        res.append(s.solve([x], [b], params))
    return res


@pytest.mark.parametrize("bcset", list(BCSETS))
@pytest.mark.parametrize("mesh", list(MESHES))
def test_cc_lap_uniform_fixed_iterations(mesh, bcset):
    ms = meshes(mesh)
    fb = setup(ms, bcset, 7)
    ig, io = solve_both(ms, OP_LAP_UNIFORM, fb, isp(30, 0.0, 0.0))
    assert ig["iterations"] == io["iterations"] == 30
    assert abs(ig["res"] - io["res"]) <= 1e-9 * io["res"], (ig, io)
    assert rel_err(fb[0][0].download(), fb[1][0].download()) < 1e-11


# (Robin is checked with the fixed budget only: with these wall conductances
# the Robin factor exceeds 1 on the fine wall cells, which makes the operator
# indefinite, and CG's iteration count to a tolerance then moves with the
# order of the floating-point sums)
@pytest.mark.parametrize("bcset", ["neumann", "dirichlet", "periodic_z", "undefined"])
@pytest.mark.parametrize("mesh", ["partial_tiles_odd", "tall"])
def test_cc_lap_uniform_to_tolerance(mesh, bcset):
    ms = meshes(mesh)
    # homogeneous BC values: with all-Neumann faces a nonzero boundary flux
    # would make the system inconsistent (the reference's mean removal comes
    # before the BC terms enter the right-hand side)
    fb = setup(ms, bcset, 8, x0=False, values=(0.0,) * 6)
    ig, io = solve_both(ms, OP_LAP_UNIFORM, fb, isp(20000, 1e-10, 1e-15))
    assert ig["exit_reason"] == io["exit_reason"]
    assert abs(ig["iterations"] - io["iterations"]) <= 1, (ig, io)
    assert rel_err(fb[0][0].download(), fb[1][0].download()) < 1e-9


@pytest.mark.parametrize("op", [OP_LAP_PROPS, OP_NRG_DIFFUSION], ids=["lap_props", "nrg_diffusion"])
@pytest.mark.parametrize("bcset", ["neumann", "periodic_y", "robin"])
def test_cc_variable_coefficient_fixed_iterations(op, bcset):
    ms = meshes("partial_tiles_odd")
    fb = setup(ms, bcset, 9)
    rng = np.random.default_rng(10)
    ks = []
    for dl in (FX, FY, FZ):
        a = 10.0 ** rng.uniform(-1, 1, ms[1].field(dl).shape)
        pair = []
        for m in ms:
            f = m.field(dl)
            f.upload(a)
            pair.append(f)
        ks.append(pair)
    ig, io = solve_both(ms, op, fb, isp(25, 0.0, 0.0), ks=ks, coeff=-0.03 if op == OP_NRG_DIFFUSION else None)
    assert abs(ig["res"] - io["res"]) <= 1e-9 * io["res"], (ig, io)
    assert rel_err(fb[0][0].download(), fb[1][0].download()) < 1e-11
