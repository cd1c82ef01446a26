"""Failure paths, made on the host (no GPU fault is ever provoked).

* A NaN in a solve's right-hand side: the reference's check_nans
  (PCG_solver_algorithm.f90:223-248) stops the run with 'Error: NaN in ...';
  the library returns MOONS_ERR_NAN from moons_pcg_solve (and the oracle
  does the same), and from moons_mhd_step when a NaN enters the state.
* A bounded in-kernel wait that runs out: moons_debug_bounded_wait waits
  1 ms on an mbarrier that nothing completes; the kernel records the site
  and returns, the call returns MOONS_ERR_CUDA naming the site, and the
  context keeps working (a solve right after it matches the oracle).
"""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from moons_b200 import configs
from tests.common import small_mesh_coords, rel_err, bc

pytestmark = pytest.mark.gpu

MOONS_ERR_CUDA = 3
MOONS_ERR_NAN = 4


def _poisson(M, m, b_arr, neumann=True):
    p = m.field(G.CC)
    p.set_bcs(bc([G.NEUMANN] * 6, all_neumann=True) if neumann else bc([G.DIRICHLET] * 6))
    b = m.field(G.CC)
    b.upload(b_arr)
    return M.PCG(m, G.OP_LAP_UNIFORM, G.PREC_LAP, [p], [p]), p, b


@pytest.mark.parametrize("where", ["interior", "ghost"])
def test_pcg_nan_rhs_returns_err_nan(where):
    cs = small_mesh_coords()
    mg_, mo = G.Mesh(*cs), O.Mesh(*cs)
    shp = mg_.field(G.CC).shape
    b = np.random.default_rng(1).standard_normal(shp)
    if where == "interior":
        b[3, 4, 2] = np.nan
    else:
        # res0 is a whole-array norm, and r = vol * (b - ...) keeps a NaN on a
        # ghost point (NaN * 0); an all-Neumann solve would zero r's ghost
        # planes first (assign_ghost_XPeriodic after the mean removal), so
        # this case uses Dirichlet faces
        b[0, 4, 2] = np.nan
    for M, m in ((G, mg_), (O, mo)):
        s, p, bf = _poisson(M, m, b, neumann=where == "interior")
        err = G.MoonsError if M is G else O.OracleError
        with pytest.raises(err) as e:
            s.solve([p], [bf], G.isp(200, 1e-10, 1e-15))
        if M is G:
            assert e.value.code == MOONS_ERR_NAN
            assert "NaN" in str(e.value)
    # the library keeps working after the error
    s, p, bf = _poisson(G, mg_, np.random.default_rng(2).standard_normal(shp))
    info = s.solve([p], [bf], G.isp(500, 1e-10, 1e-15))
    assert info["exit_reason"] == 1


def test_mhd_step_nan_state_returns_err_nan():
    sim = configs.make(G, configs.ldc, seed=0, n=8)
    u = sim.download(G.MHD_U, 0)
    u[4, 4, 4] = np.nan
    sim.upload(G.MHD_U, 0, u)
    with pytest.raises(G.MoonsError) as e:
        sim.step(1)
    assert e.value.code == MOONS_ERR_NAN


def test_bounded_wait_runs_out_and_context_survives():
    with pytest.raises(G.MoonsError) as e:
        G.debug_bounded_wait(1_000_000)  # 1 ms
    assert e.value.code == MOONS_ERR_CUDA
    assert "site 900" in str(e.value)
    with pytest.raises(G.MoonsError):
        G.debug_bounded_wait(0)  # limits outside (0, 1 s] are refused
    # the context still runs kernels: a solve matches the oracle
    cs = small_mesh_coords()
    b = np.random.default_rng(3).standard_normal(G.Mesh(*cs).field(G.CC).shape)
    out = []
    for M in (G, O):
        s, p, bf = _poisson(M, M.Mesh(*cs), b)
        out.append((s.solve([p], [bf], G.isp(500, 1e-10, 1e-15)), p.download()))
    assert abs(out[0][0]["iterations"] - out[1][0]["iterations"]) <= 1
    assert rel_err(out[0][1], out[1][1]) < 1e-8
