"""moons_clean_div -- the clean_div call site of the reference
(clean_divergence.f90:37-59) -- against the oracle's restatement on the same
inputs: the projected field and the potential, with Neumann walls and with
periodic faces."""
import numpy as np
import pytest

import oracle.oracle as O
from moons_b200 import capi as G
from tests import clean_div_case as CD
from tests.common import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("periodic", [False, True])
def test_clean_div_matches_oracle(periodic):
    out = []
    for M in (G, O):
        m, pcg, X, Xs, phi, tF, tcc = CD.build(M, periodic)
        info = M.clean_div(pcg, X, Xs, phi, 100.0, tF, tcc, G.isp(5000, 1e-12, 1e-300))
        out.append((info, [x.download() for x in X], phi.download(), m, X, Xs))
    (ig, xg, pg, mg, Xg, Xsg), (io, xo, po, *_) = out
    assert ig["exit_reason"] == io["exit_reason"] == 1, (ig, io)
    assert abs(ig["iterations"] - io["iterations"]) <= 1, (ig, io)
    for a, b in zip(xg, xo):
        assert rel_err(a, b) < 1e-9
    pi = pg[1:-1, 1:-1, 1:-1] - pg[1:-1, 1:-1, 1:-1].mean()
    qi = po[1:-1, 1:-1, 1:-1] - po[1:-1, 1:-1, 1:-1].mean()
    assert rel_err(pi, qi) < 1e-8
    if periodic:
        d0 = np.linalg.norm(CD.interior_div(G, mg, Xsg))
        assert np.linalg.norm(CD.interior_div(G, mg, Xg)) < 1e-9 * d0
