"""The oracle's clean_div (clean_divergence.f90:37-59) on the CPU: with
periodic faces the projected field is divergence-free to the solver's
tolerance."""
import numpy as np

import oracle.oracle as O
from moons_b200 import capi as G
from tests import clean_div_case as CD


def test_oracle_clean_div_removes_the_divergence():
    m, pcg, X, Xs, phi, tF, tcc = CD.build(O, periodic=True)
    d0 = np.linalg.norm(CD.interior_div(O, m, Xs))
    info = O.clean_div(pcg, X, Xs, phi, 100.0, tF, tcc, G.isp(5000, 1e-12, 1e-300))
    assert info["exit_reason"] == 1, info
    d1 = np.linalg.norm(CD.interior_div(O, m, X))
    assert d1 < 1e-9 * d0, (d0, d1)
