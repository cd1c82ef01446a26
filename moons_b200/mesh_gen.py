"""Node-coordinate generators of the reference (host side of row a2).

The Fortran host builds ``hn`` itself and passes it through the C-ABI; these
functions restate the generators the configurations use so Python callers
(tests, bench) produce the same coordinates:

* ``uniform``       -- uniform_func (HW/grid/coordinate_distribution_funcs.f90:34-56)
* ``roberts_both``  -- robertsBoth_func = transformation2 with alpha=0.5
                       (coordinate_distribution_funcs.f90:192-248, :325-331)
* ``add_ghost_nodes`` -- add_ghost_nodes_c (HW/grid/coordinates_extend.f90:529-538)
"""
from __future__ import annotations

import numpy as np


def uniform(hmin: float, hmax: float, n: int) -> np.ndarray:
    dh = (hmax - hmin) / float(n)
    return np.array([hmin + float(i) * dh for i in range(n + 1)], dtype=np.float64)


def roberts(hmin: float, hmax: float, n: int, alpha: float, beta: float) -> np.ndarray:
    a, b = alpha, beta
    g = (b + 1.0) / (b - 1.0)
    dh = (hmax - hmin) / float(n)
    hnbar = np.array([hmin + float(i) * dh for i in range(n + 1)])
    hnbar = (hnbar - hmin) / (hmax - hmin)
    e = g ** ((hnbar - a) / (1.0 - a))
    hn = ((b + 2.0 * a) * e - b + 2.0 * a) / ((2.0 * a + 1.0) * (1.0 + e))
    return hmin + (hmax - hmin) * hn


def roberts_both(hmin: float, hmax: float, n: int, beta: float) -> np.ndarray:
    return roberts(hmin, hmax, n, 0.5, beta)


def add_ghost_nodes(hn: np.ndarray) -> np.ndarray:
    hn = np.asarray(hn, dtype=np.float64)
    return np.concatenate([[hn[0] - (hn[1] - hn[0])], hn, [hn[-1] + (hn[-1] - hn[-2])]])


def with_ghosts(hn: np.ndarray) -> np.ndarray:
    return add_ghost_nodes(hn)
