"""A clean_div (clean_divergence.f90:37-59) case for the CPU and GPU tests:
Xstar i.i.d. N(0,1) on the three face fields of a stretched mesh, the
projection potential phi with Neumann walls (all-Neumann: the solver
removes the right-hand side's mean) or periodic faces, scale = 1/dt."""
import numpy as np

from moons_b200 import capi as G
from tests.common import small_mesh_coords, bc

DLS = (G.FX, G.FY, G.FZ)


def build(backend, periodic: bool, seed: int = 3):
    # a periodic axis needs equal end cells: uniform there
    cs = small_mesh_coords(n=(12, 10, 8), stretched=not periodic)
    m = backend.Mesh(*cs)
    rng = np.random.default_rng(seed)
    if periodic:
        types_x = [G.PERIODIC] * 6
        types_p = [G.PERIODIC] * 6
    else:
        types_x = [G.DIRICHLET] * 6
        types_p = [G.NEUMANN] * 6
    X, Xs, tF = [], [], []
    for dl in DLS:
        x, xs, t = m.field(dl), m.field(dl), m.field(dl)
        for f in (x, xs):
            f.set_bcs(bc(types_x))
        xs.upload(rng.standard_normal(xs.shape))
        xs.apply_bcs()  # boundary values consistent with the BCs, as a solve leaves them
        x.fill(0.0)
        X.append(x)
        Xs.append(xs)
        tF.append(t)
    phi, tcc = m.field(G.CC), m.field(G.CC)
    phi.set_bcs(bc(types_p, all_neumann=True))
    phi.fill(0.0)
    pcg = backend.PCG(m, G.OP_LAP_UNIFORM, G.PREC_LAP, [phi], [phi])
    return m, pcg, X, Xs, phi, tF, tcc


def interior_div(backend, m, X):
    d = m.field(G.CC)
    backend.div(d, *X)
    return d.download()[1:-1, 1:-1, 1:-1]
