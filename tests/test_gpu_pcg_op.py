"""moons_pcg_apply_op -- the solver's operator as the abstract op_SF / op_VF
(matrix_free_operators_interfaces.f90:14-60) binds it, operator_explicit of
matrix_free_operators.f90 -- against the oracle's PCG::apply_operator on the
same fields, for every operator of the path: Lap_uniform, Lap_nonuniform_props, nrg_diffusion, mom_diffusion and
ind_diffusion, with ghost values taken as they are (random), on a stretched
mesh with odd extents."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200.capi import (CC, FX, FY, FZ, EX, EY, EZ, DIRICHLET, NEUMANN, OP_LAP_UNIFORM, OP_LAP_PROPS,
                             OP_MOM_DIFFUSION, OP_IND_DIFFUSION, OP_NRG_DIFFUSION, PREC_LAP, PREC_MOM, PREC_IND)
from tests.common import small_mesh_coords, rel_err, bc

pytestmark = pytest.mark.gpu


def pair(ms, dl, a):
    g, o = ms[0].field(dl), ms[1].field(dl)
    g.upload(a)
    o.upload(a)
    return g, o


CASES = {
    "lap_uniform_cc": (OP_LAP_UNIFORM, PREC_LAP, [CC], None, None),
    "lap_props": (OP_LAP_PROPS, PREC_LAP, [CC], [FX, FY, FZ], None),
    "nrg_diffusion": (OP_NRG_DIFFUSION, PREC_LAP, [CC], [FX, FY, FZ], -0.02),
    "mom_diffusion": (OP_MOM_DIFFUSION, PREC_MOM, [FX, FY, FZ], None, -0.03),
    "ind_diffusion": (OP_IND_DIFFUSION, PREC_IND, [FX, FY, FZ], [EX, EY, EZ], 0.05),
}


@pytest.mark.parametrize("case", list(CASES))
def test_apply_op_matches_oracle(case):
    op, prec, dls, kdls, coeff = CASES[case]
    cs = small_mesh_coords()
    ms = G.Mesh(*cs), O.Mesh(*cs)
    rng = np.random.default_rng(11)
    xs, outs = [], []
    for c, dl in enumerate(dls):
        shp = ms[1].field(dl).shape
        x = pair(ms, dl, rng.standard_normal(shp))
        types = [DIRICHLET] * 6
        types[2 * (c % 3)] = NEUMANN
        for f in x:
            f.set_bcs(bc(types))
        xs.append(x)
        outs.append(pair(ms, dl, np.zeros(shp)))
    ks = None
    if kdls:
        ks = [pair(ms, dl, 10.0 ** rng.uniform(-1, 1, ms[1].field(dl).shape)) for dl in kdls]
    sg = G.PCG(ms[0], op, prec, [x[0] for x in xs], [x[0] for x in xs], [k[0] for k in ks] if ks else None)
    so = O.PCG(ms[1], op, prec, [x[1] for x in xs], [x[1] for x in xs], [k[1] for k in ks] if ks else None)
    if coeff is not None:
        sg.update_mfp(coeff, True)
        so.update_mfp(coeff, True)
    for _ in range(2):  # twice: the scratch the operator uses carries nothing over
        sg.apply_op([o[0] for o in outs], [x[0] for x in xs])
        so.apply_op([o[1] for o in outs], [x[1] for x in xs])
        for g, o in outs:
            a, b = g.download(), o.download()
            assert rel_err(a, b) < 1e-12, (case, rel_err(a, b))
    # a field of another layout is refused
    wrong = ms[0].field(EZ if dls[0] != EZ else CC)
    with pytest.raises(G.MoonsError):
        sg.apply_op([wrong] * len(dls), [x[0] for x in xs])
