"""Mesh generation of the reference, host side.

The Fortran host builds the node coordinates ``hn`` itself and passes them
through the C-ABI; this module restates its generators so Python callers
(tests, bench, case presets) produce the same coordinates, the same
three-mesh layouts (fluid, conductor, induction with vacuum) and the same
sub-domain index ranges the GPU path embeds and extracts with.

Coordinate distributions (code/handwritten/grid/coordinate_distribution_funcs.f90):

* ``uniform`` / ``linspace``        -- uniform_func / linspace_func (:34-81)
* ``uniform_left`` / ``uniform_right`` -- uniformDirection_func (:83-143)
* ``roberts_left``   -- transformation1, clustered at hmin (:145-190, :309-315)
* ``roberts_right``  -- transformation2 with alpha = 0, clustered at hmax (:192-248, :317-323)
* ``roberts_both``   -- transformation2 with alpha = 0.5 (:325-331)
* ``cluster``        -- transformation3, clustered about yc (:250-307, :333-339)

Iterated forms that add points until the neighbour spacing ratio is at most
``max_mesh_stretch_ratio`` (coordinate_distribution_funcs_iterate.f90:64-152),
boundary-layer stretching parameters (coordinate_stretch_parameters.f90:16-135),
the Newton match of a Roberts parameter to a given end spacing
(coordinate_stretch_param_match.f90:37-265, newtonT2 :181-234), grid
construction and extension (grid/grid_init.f90:22-79,
grid/grid_continue.f90:1-317), the segment list of
a mesh (mesh_params/segment_extend.f90, mesh_params_extend.f90) and its
generator (mesh/generate_mesh_generic.f90:20-97), and the index overlap of
two meshes (sub_domain/overlap_extend.f90:204-290, 364-380).

The reference stops the program on bad input; these functions raise
ValueError instead.
"""
from __future__ import annotations

import copy
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

_EPS = float(np.finfo(np.float64).eps)   # machine_epsilon = epsilon(1.0_cp)
_TOL = 1e-12                             # coordinate_distribution_funcs.f90: tol


# ---- coordinate distributions ------------------------------------------------

def uniform(hmin: float, hmax: float, n: int) -> np.ndarray:
    """uniform_func: n cells, n + 1 nodes; n = 0 allowed when hmin == hmax."""
    if n < 0:
        raise ValueError("N < 0 in uniform")
    if n == 0:
        if abs(hmax - hmin) < _TOL:
            return np.array([hmin], dtype=np.float64)
        raise ValueError("N = 0 but hmin != hmax in uniform")
    dh = (hmax - hmin) / float(n)
    return np.array([hmin + float(i) * dh for i in range(n + 1)], dtype=np.float64)


def linspace(hmin: float, hmax: float, n: int) -> np.ndarray:
    dh = (hmax - hmin) / float(n)
    return np.array([hmin + float(i) * dh for i in range(n + 1)], dtype=np.float64)


def _uniform_direction(hstart: float, dh: float, n: int, d: int) -> np.ndarray:
    if n < 0:
        raise ValueError("N < 0 in uniformDirection")
    if n == 0:
        if dh < _TOL:
            return np.array([hstart], dtype=np.float64)
        raise ValueError("N = 0 but dh > tol in uniformDirection")
    hn = np.array([hstart + (float(d) * float(i)) * dh for i in range(n + 1)], dtype=np.float64)
    return hn[::-1].copy() if d == -1 else hn


def uniform_left(hstart: float, dh: float, n: int) -> np.ndarray:
    """n cells of size dh ending at hstart."""
    return _uniform_direction(hstart, dh, n, -1)


def uniform_right(hstart: float, dh: float, n: int) -> np.ndarray:
    """n cells of size dh starting at hstart."""
    return _uniform_direction(hstart, dh, n, 1)


def _unit(hmin: float, hmax: float, n: int) -> np.ndarray:
    dh = (hmax - hmin) / float(n)
    hnbar = np.array([hmin + float(i) * dh for i in range(n + 1)])
    return (hnbar - hmin) / (hmax - hmin)


def _insist(h: np.ndarray, increasing: bool, caller: str):
    for i in range(len(h) - 2):
        R = (h[i + 2] - h[i + 1]) / (h[i + 1] - h[i])
        if (R < 1.0) if increasing else (R > 1.0):
            kind = "increasing" if increasing else "decreasing"
            raise ValueError(f"coordinates not monotonically {kind} in {caller} (R = {R})")


def roberts_left_raw(hmin: float, hmax: float, n: int, beta: float) -> np.ndarray:
    """transformation1 (alpha = 1): spacing grows away from hmin."""
    a, b = 1.0, beta
    g = (b + 1.0) / (b - 1.0)
    x = _unit(hmin, hmax, n)
    hn = np.array([((b + a) - (b - a) * g ** (a - xi)) / (g ** (a - xi) + a) for xi in x])
    _insist(hn, True, "transformation1")
    return hmin + (hmax - hmin) * hn


def roberts(hmin: float, hmax: float, n: int, alpha: float, beta: float) -> np.ndarray:
    """transformation2 (Roberts, alpha in [0, 0.5])."""
    a, b = alpha, beta
    g = (b + 1.0) / (b - 1.0)
    x = _unit(hmin, hmax, n)
    e = np.array([g ** ((xi - a) / (1.0 - a)) for xi in x])
    hn = ((b + 2.0 * a) * e - b + 2.0 * a) / ((2.0 * a + 1.0) * (1.0 + e))
    if abs(alpha) < 1e-10:
        _insist(hn, False, "transformation2")
    return hmin + (hmax - hmin) * hn


def roberts_left(hmin: float, hmax: float, n: int, beta: float) -> np.ndarray:
    return roberts_left_raw(hmin, hmax, n, beta)


def roberts_right(hmin: float, hmax: float, n: int, beta: float) -> np.ndarray:
    return roberts(hmin, hmax, n, 0.0, beta)


def roberts_both(hmin: float, hmax: float, n: int, beta: float) -> np.ndarray:
    return roberts(hmin, hmax, n, 0.5, beta)


def cluster(hmin: float, hmax: float, n: int, yc: float, tau: float) -> np.ndarray:
    """transformation3: points clustered about yc with strength tau."""
    a, c = 1.0, 2.0
    x = _unit(hmin, hmax, n)
    d = yc / (hmax - hmin)
    e = math.exp(tau)
    B = a / (c * tau) * math.log((a + (e - a) * d) / (a + (a / e - a) * d))
    hn = np.array([d * (a + math.sinh(tau * (xi - B)) / math.sinh(tau * B)) for xi in x])
    return hmin + (hmax - hmin) * hn


# ---- mesh quality and the iterated distributions ------------------------------

@dataclass
class MeshQuality:
    """mesh_quality_params (mesh_quality_params_extend.f90:18-33): with
    auto_find_N the generators may add up to N_max_points_add points until
    no two neighbouring cells differ in size by more than
    max_mesh_stretch_ratio; without it they run once.  The default is the
    reference's manual_MQP (no search)."""
    auto_find_N: bool = False
    max_mesh_stretch_ratio: float = 1.0
    N_max_points_add: int = 1

    @property
    def N_iter(self) -> int:
        return self.N_max_points_add + 1 if self.auto_find_N else 1


def needs_more_points(hn: np.ndarray, mqp: MeshQuality) -> bool:
    """needs_more_points_func: largest neighbour spacing ratio above the limit."""
    hn = np.asarray(hn, dtype=np.float64)
    if len(hn) <= 2:
        return False
    dhn = np.diff(hn)
    R = np.maximum(dhn[:-1] / dhn[1:], dhn[1:] / dhn[:-1])
    return bool(R.max() > mqp.max_mesh_stretch_ratio)


def _iterate(f, n: int, mqp: MeshQuality) -> np.ndarray:
    hn = None
    temp = n
    for _ in range(mqp.N_iter):
        hn = f(temp)
        if needs_more_points(hn, mqp):
            temp += 1
        else:
            break
    if hn is None:
        raise ValueError("mesh quality parameters with N_iter = 0 generate no coordinates")
    return hn


def roberts_left_iterate(hmin, hmax, n, beta, mqp: MeshQuality):
    return _iterate(lambda m: roberts_left(hmin, hmax, m, beta), n, mqp)


def roberts_right_iterate(hmin, hmax, n, beta, mqp: MeshQuality):
    return _iterate(lambda m: roberts_right(hmin, hmax, m, beta), n, mqp)


def roberts_both_iterate(hmin, hmax, n, beta, mqp: MeshQuality):
    return _iterate(lambda m: roberts_both(hmin, hmax, m, beta), n, mqp)


def cluster_iterate(hmin, hmax, n, yc, tau, mqp: MeshQuality):
    return _iterate(lambda m: cluster(hmin, hmax, m, yc, tau), n, mqp)


# ---- boundary-layer stretching parameters -------------------------------------

def roberts_bl_1d(delta: float, h: float) -> float:
    """RobertsBL1D: beta for a boundary layer of thickness delta on a length h
    (Tannehill et al., Computational Fluid Mechanics and Heat Transfer, 5.6);
    1000 (nearly uniform) when delta >= 0.99 h."""
    if delta < h * 0.99:
        return (1.0 - delta / h) ** (-0.5)
    return 1000.0


def hartmann_bl_1d(Ha: float, hmin: float, hmax: float) -> float:
    if Ha < 1e-10:
        raise ValueError("Hartmann number is nearly zero in HartmannBL")
    return roberts_bl_1d((hmax - hmin) / Ha, hmax - hmin)


def reynolds_bl_1d(Re: float, hmin: float, hmax: float) -> float:
    if Re < 1e-10:
        raise ValueError("Reynolds number is nearly zero in ReynoldsBL")
    return roberts_bl_1d((hmax - hmin) / math.sqrt(Re), hmax - hmin)


def re_ha_bl_1d(Re: float, Ha: float, hmin: float, hmax: float) -> float:
    """Re_Ha_BL_1D: the smaller of the Reynolds (L/sqrt(Re)) and Hartmann
    (L/Ha) layer parameters."""
    return min(reynolds_bl_1d(Re, hmin, hmax), hartmann_bl_1d(Ha, hmin, hmax))


# ---- Roberts parameter matched to an end spacing ------------------------------

def _t2_h(beta, alpha, i, n):
    a, b = alpha, beta
    g = (b + 1.0) / (b - 1.0)
    t = (float(i) / float(n) - a) / (1.0 - a)
    return ((b + 2.0 * a) * g ** t - b + 2.0 * a) / ((2.0 * a + 1.0) * (1.0 + g ** t))


def _t2_prime_h(beta, alpha, i, n):
    # the reference's closed form of the beta-derivative, kept as written
    a, b = alpha, beta
    g = (b + 1.0) / (b - 1.0)
    t = (float(i) / float(n) - a) / (1.0 - a)
    return -(-b ** 2.0 * g ** (2.0 * t) + b ** 2.0 + 4.0 * b * g ** t * t
             + g ** (2.0 * t) - 1.0) / ((2.0 * a + 1.0) * (b - 1.0) * (b + 1.0) * (g ** t + 1.0) ** 2.0)


def _root_near_hmax(beta, hmin, hmax, alpha, n, dh):
    return _t2_h(beta, alpha, n, n) - _t2_h(beta, alpha, n - 1, n) - dh / (hmax - hmin)


def _prime_near_hmax(beta, alpha, n):
    return _t2_prime_h(beta, alpha, n, n) - _t2_prime_h(beta, alpha, n - 1, n)


def _root_near_hmin(beta, hmin, hmax, alpha, n, dh):
    return _t2_h(beta, alpha, 1, n) - _t2_h(beta, alpha, 0, n) - dh / (hmax - hmin)


def _prime_near_hmin(beta, alpha, n):
    return _t2_prime_h(beta, alpha, 1, n) - _t2_prime_h(beta, alpha, 0, n)


#: set by _newton_t2 when the match did not converge and beta fell back to 1.1
#: (the reference writes the file 'mesh_generation_error' in that case)
last_match_error: Optional[str] = None


def _newton_t2(root, prime, hmin, hmax, alpha, n, dh) -> float:
    """newtonT2: Newton iteration from beta = 1 + 1e-10 to |f| < 10 eps;
    stops when beta > 1000; a beta below 1 + 1e-10 becomes 1.1; a NaN or a
    residual still above the tolerance falls back to beta = 1.1.  The
    reference runs up to 10^6 steps; an iteration that revisits a beta is
    periodic and can only end in the fallback, so it stops there."""
    global last_match_error
    last_match_error = None
    maxiter = 1000000
    tol = 10.0 * _EPS
    beta_low = 1.0 + 1e-10
    beta = 1.0 + 1e-10
    fbeta = float("nan")
    seen = set()
    with np.errstate(all="ignore"):
        for _ in range(maxiter):
            fbeta = root(beta, hmin, hmax, alpha, n, dh)
            fprime = prime(beta, alpha, n)
            if abs(fbeta) < tol:
                break
            if beta > 1000.0:
                break
            if beta < beta_low:
                beta = 1.1
                break
            if beta in seen:
                fbeta = float("inf")  # periodic: the loop would end without success
                break
            seen.add(beta)
            beta = beta - fbeta / fprime
            if math.isnan(beta):
                break
    if math.isnan(beta) or abs(fbeta) > tol:
        last_match_error = f"newtonT2 not converged: beta = {beta}, fbeta = {fbeta}, tol = {tol}"
        beta = 1.1
    return beta


def beta_dh_small(hmin: float, hmax: float, n: int, dh: float) -> float:
    """Roberts (alpha = 0) parameter whose cell next to hmax has size dh."""
    return _newton_t2(_root_near_hmax, _prime_near_hmax, hmin, hmax, 0.0, n, dh)


def beta_dh_big(hmin: float, hmax: float, n: int, dh: float) -> float:
    """Roberts (alpha = 0) parameter whose cell next to hmin has size dh."""
    return _newton_t2(_root_near_hmin, _prime_near_hmin, hmin, hmax, 0.0, n, dh)


def beta_dh_both(hmin: float, hmax: float, n: int, dh: float) -> float:
    """Two-sided Roberts (alpha = 0.5) parameter whose end cells have size dh."""
    return _newton_t2(_root_near_hmax, _prime_near_hmax, hmin, hmax, 0.5, n, dh)


# ---- ghost nodes and coordinate properties ------------------------------------

def add_ghost_nodes(hn: np.ndarray) -> np.ndarray:
    """add_ghost_nodes_c (coordinates_extend.f90:529-538): one node beyond
    each end at the end spacing."""
    hn = np.asarray(hn, dtype=np.float64)
    if len(hn) < 2:
        raise ValueError("trying to add ghost points to a single point")
    return np.concatenate([[hn[0] - (hn[1] - hn[0])], hn, [hn[-1] + (hn[-1] - hn[-2])]])


def with_ghosts(hn: np.ndarray) -> np.ndarray:
    return add_ghost_nodes(hn)


def _prepend_ghost(hn):
    if len(hn) < 2:
        raise ValueError("trying to prepend a ghost point to a single point")
    return np.concatenate([[hn[0] - (hn[1] - hn[0])], hn])


def _append_ghost(hn):
    if len(hn) < 2:
        raise ValueError("trying to append a ghost point to a single point")
    return np.concatenate([hn, [hn[-1] + (hn[-1] - hn[-2])]])


def _hmin(hn):
    return hn[1] if len(hn) > 2 else hn[0]


def _hmax(hn):
    return hn[-2] if len(hn) > 2 else hn[-1]


def _dh_first(hn):
    return hn[1] - hn[0]


def _dh_last(hn):
    return hn[-1] - hn[-2]


# ---- grids: base distributions and extensions ---------------------------------

class Grid:
    """Three node-coordinate arrays with one ghost node per side (the
    reference's grid with coordinates c(1:3)); ``hn[d]`` is None until a
    base distribution sets direction d."""

    def __init__(self):
        self.hn: List[Optional[np.ndarray]] = [None, None, None]

    def coords(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        if any(h is None for h in self.hn):
            raise ValueError("grid direction without coordinates")
        return tuple(h.copy() for h in self.hn)

    def cells(self) -> Tuple[int, int, int]:
        """Physical cells per direction (ghost cells excluded)."""
        return tuple(len(h) - 3 for h in self.hn)

    def _c(self, d):
        h = self.hn[d - 1]
        if h is None:
            raise ValueError(f"direction {d} has no base distribution to extend")
        return h

    # base distributions (grid_init.f90:22-79)
    def grid_uniform(self, hmin, hmax, n, d):
        self.hn[d - 1] = add_ghost_nodes(uniform(hmin, hmax, n))

    def grid_roberts_l(self, hmin, hmax, n, beta, d, mqp):
        self.hn[d - 1] = add_ghost_nodes(roberts_left_iterate(hmin, hmax, n, beta, mqp))

    def grid_roberts_r(self, hmin, hmax, n, beta, d, mqp):
        self.hn[d - 1] = add_ghost_nodes(roberts_right_iterate(hmin, hmax, n, beta, mqp))

    def grid_roberts_b(self, hmin, hmax, n, beta, d, mqp):
        self.hn[d - 1] = add_ghost_nodes(roberts_both_iterate(hmin, hmax, n, beta, mqp))

    def grid_cluster(self, hmin, hmax, n, yc, tau, d, mqp):
        self.hn[d - 1] = add_ghost_nodes(cluster_iterate(hmin, hmax, n, yc, tau, mqp))

    # extensions (grid_continue.f90)
    def _prepend(self, d, b):
        # process_prepend: drop the ghost and hmin, put b (ending at hmin) in front
        a = self._c(d)[2:]
        self.hn[d - 1] = _prepend_ghost(np.concatenate([b, a]))

    def _append(self, d, b):
        # process_append: drop hmax and the ghost, put b (starting at hmax) behind
        a = self._c(d)[:-2]
        self.hn[d - 1] = _append_ghost(np.concatenate([a, b]))

    @staticmethod
    def _check_n(n, caller):
        if not n > 0:
            raise ValueError(f"N is not > 0 in {caller}")

    def _matched(self, beta_fn, dist_fn, lo, hi, n, dh, mqp):
        # the reference's loop: N_final takes the point count of the last try
        # (one more than its cells) before adding a point
        b = None
        n_final = n
        for _ in range(mqp.N_iter):
            beta = beta_fn(lo, hi, n_final, dh)
            b = dist_fn(lo, hi, n_final, beta)
            n_final = len(b)
            if needs_more_points(b, mqp):
                n_final += 1
            else:
                break
        if b is None:
            raise ValueError("mesh quality parameters with N_iter = 0 generate no coordinates")
        return b

    def ext_prep_uniform(self, n, d):
        self._check_n(n, "ext_prep_uniform_IO")
        h = self._c(d)
        self._prepend(d, uniform_left(_hmin(h), _dh_first(h), n))

    def ext_prep_roberts_l(self, L, n, d, mqp):
        self._check_n(n, "ext_prep_Roberts_L_IO")
        h = self._c(d)
        hmin, dh = _hmin(h), _dh_first(h)
        self._prepend(d, self._matched(beta_dh_small, roberts_left, hmin - L, hmin, n, dh, mqp))

    def ext_prep_roberts_r(self, L, n, d, mqp):
        self._check_n(n, "ext_prep_Roberts_R_IO")
        h = self._c(d)
        hmin, dh = _hmin(h), _dh_first(h)
        self._prepend(d, self._matched(beta_dh_small, roberts_right, hmin - L, hmin, n, dh, mqp))

    def ext_prep_roberts_b(self, L, n, d, mqp):
        self._check_n(n, "ext_prep_Roberts_B_IO")
        h = self._c(d)
        hmin, dh = _hmin(h), _dh_first(h)
        self._prepend(d, self._matched(beta_dh_both, roberts_both, hmin - L, hmin, n, dh, mqp))

    def ext_prep_roberts_c2f(self, L, n, d, mqp):
        self._check_n(n, "ext_prep_Roberts_C2F_IO")
        h = self._c(d)
        hmin, dh = _hmin(h), _dh_first(h)
        self._prepend(d, self._matched(beta_dh_big, roberts_left, hmin - L, hmin, n, dh, mqp))

    def ext_app_uniform(self, n, d):
        self._check_n(n, "ext_app_uniform_IO")
        h = self._c(d)
        self._append(d, uniform_right(_hmax(h), _dh_last(h), n))

    def ext_app_roberts_l(self, L, n, d, mqp):
        self._check_n(n, "ext_app_Roberts_L_IO")
        h = self._c(d)
        hmax, dh = _hmax(h), _dh_last(h)
        self._append(d, self._matched(beta_dh_small, roberts_left, hmax, hmax + L, n, dh, mqp))

    def ext_app_roberts_r(self, L, n, d, mqp):
        self._check_n(n, "ext_app_Roberts_R_IO")
        h = self._c(d)
        hmax, dh = _hmax(h), _dh_last(h)
        self._append(d, self._matched(beta_dh_small, roberts_right, hmax, hmax + L, n, dh, mqp))

    def ext_app_roberts_b(self, L, n, d, mqp):
        self._check_n(n, "ext_app_Roberts_B_IO")
        h = self._c(d)
        hmax, dh = _hmax(h), _dh_last(h)
        self._append(d, self._matched(beta_dh_both, roberts_both, hmax, hmax + L, n, dh, mqp))

    def ext_app_roberts_c2f(self, L, n, d, mqp):
        self._check_n(n, "ext_app_Roberts_C2F_IO")
        h = self._c(d)
        hmax, dh = _hmax(h), _dh_last(h)
        self._append(d, self._matched(beta_dh_big, roberts_right, hmax, hmax + L, n, dh, mqp))

    # both sides (grid_continue.f90:38-75)
    def ext_uniform(self, n, d):
        self.ext_prep_uniform(n, d)
        self.ext_app_uniform(n, d)

    def ext_roberts_near(self, L, n, d, mqp):
        self.ext_prep_roberts_r(L, n, d, mqp)
        self.ext_app_roberts_l(L, n, d, mqp)

    def ext_roberts_far(self, L, n, d, mqp):
        self.ext_prep_roberts_l(L, n, d, mqp)
        self.ext_app_roberts_r(L, n, d, mqp)

    def ext_roberts_b(self, L, n, d, mqp):
        self.ext_prep_roberts_b(L, n, d, mqp)
        self.ext_app_roberts_b(L, n, d, mqp)


# ---- segments, mesh parameters and the generic generator ----------------------

@dataclass
class Segment:
    """One base or extension segment of a mesh (segment.f90): the
    distribution's name as the reference spells it, the direction (1..3),
    the cells, the bounds (base) or the length (extension), the boundary-layer
    buffer and the cluster parameters."""
    dir: int
    distribution: str
    n_cells: int
    hmin: float = 0.0
    hmax: float = 0.0
    L: float = 0.0
    buffer: float = 0.0
    tau: float = 0.0
    yc: float = 0.0


def seg_1d(dir: int, distribution: str, n_cells: int, *args: float) -> Segment:
    """seg_1d overloads (segment_extend.f90): (hmin, hmax, buffer) for a base
    segment, (L, buffer) for an extension, or the cell count alone (buffer 1)."""
    if len(args) == 3:
        return Segment(dir, distribution, n_cells, hmin=args[0], hmax=args[1], buffer=args[2])
    if len(args) == 2:
        return Segment(dir, distribution, n_cells, L=args[0], buffer=args[1])
    if len(args) == 0:
        return Segment(dir, distribution, n_cells, buffer=1.0)
    raise ValueError("seg_1d takes (hmin, hmax, buffer), (L, buffer) or nothing after the cell count")


@dataclass
class MeshParams:
    """mesh_params: the mesh quality settings and the base and extension
    segments, applied in the order they were added."""
    mqp: MeshQuality = field(default_factory=MeshQuality)
    s_base: List[Segment] = field(default_factory=list)
    s_ext: List[Segment] = field(default_factory=list)

    def add_base(self, s: Segment) -> "MeshParams":
        self.s_base.append(copy.copy(s))
        return self

    def add_ext(self, s: Segment) -> "MeshParams":
        self.s_ext.append(copy.copy(s))
        return self

    def copy(self) -> "MeshParams":
        return copy.deepcopy(self)


_BASE = ("grid_uniform", "grid_Roberts_L", "grid_Roberts_R", "grid_Roberts_B", "grid_cluster")
_EXT = ("ext_uniform_IO", "ext_Roberts_near_IO", "ext_Roberts_far_IO", "ext_Roberts_B_IO",
        "ext_prep_uniform_IO", "ext_prep_Roberts_L_IO", "ext_prep_Roberts_R_IO", "ext_prep_Roberts_B_IO",
        "ext_app_uniform_IO", "ext_app_Roberts_L_IO", "ext_app_Roberts_R_IO", "ext_app_Roberts_B_IO",
        "ext_app_Roberts_C2F_IO", "ext_prep_Roberts_C2F_IO")


def generate_mesh_generic(mp: MeshParams, Re: float, Ha: float, caller: str = "") -> Grid:
    """generate_mesh_generic: every base segment sets its direction, then
    every extension segment extends its direction, in order; segments with
    no cells are skipped.  Each segment's Roberts parameter is
    Re_Ha_BL_1D(Re*buffer, Ha*buffer, hmin, hmax), evaluated for every
    segment as the reference does (so Re and Ha must be nonzero)."""
    g = Grid()
    q = mp.mqp
    for s in mp.s_base:
        beta = re_ha_bl_1d(Re * s.buffer, Ha * s.buffer, s.hmin, s.hmax)
        if s.n_cells <= 0:
            continue
        a, b, n, d = s.hmin, s.hmax, s.n_cells, s.dir
        if s.distribution == "grid_uniform":
            g.grid_uniform(a, b, n, d)
        elif s.distribution == "grid_Roberts_L":
            g.grid_roberts_l(a, b, n, beta, d, q)
        elif s.distribution == "grid_Roberts_R":
            g.grid_roberts_r(a, b, n, beta, d, q)
        elif s.distribution == "grid_Roberts_B":
            g.grid_roberts_b(a, b, n, beta, d, q)
        elif s.distribution == "grid_cluster":
            g.grid_cluster(a, b, n, s.yc, s.tau, d, q)
        else:
            raise ValueError(f"bad distribution in mesh base {caller} for mesh {s.distribution}")
    for s in mp.s_ext:
        re_ha_bl_1d(Re * s.buffer, Ha * s.buffer, s.hmin, s.hmax)
        if s.n_cells <= 0:
            continue
        L, n, d, dist = s.L, s.n_cells, s.dir, s.distribution
        if dist == "ext_uniform_IO":
            g.ext_uniform(n, d)
        elif dist == "ext_Roberts_near_IO":
            g.ext_roberts_near(L, n, d, q)
        elif dist == "ext_Roberts_far_IO":
            g.ext_roberts_far(L, n, d, q)
        elif dist == "ext_Roberts_B_IO":
            g.ext_roberts_b(L, n, d, q)
        elif dist == "ext_prep_uniform_IO":
            g.ext_prep_uniform(n, d)
        elif dist == "ext_prep_Roberts_L_IO":
            g.ext_prep_roberts_l(L, n, d, q)
        elif dist == "ext_prep_Roberts_R_IO":
            g.ext_prep_roberts_r(L, n, d, q)
        elif dist == "ext_prep_Roberts_B_IO":
            g.ext_prep_roberts_b(L, n, d, q)
        elif dist == "ext_app_uniform_IO":
            g.ext_app_uniform(n, d)
        elif dist == "ext_app_Roberts_L_IO":
            g.ext_app_roberts_l(L, n, d, q)
        elif dist == "ext_app_Roberts_R_IO":
            g.ext_app_roberts_r(L, n, d, q)
        elif dist == "ext_app_Roberts_B_IO":
            g.ext_app_roberts_b(L, n, d, q)
        elif dist == "ext_app_Roberts_C2F_IO":
            g.ext_app_roberts_c2f(L, n, d, q)
        elif dist == "ext_prep_Roberts_C2F_IO":
            g.ext_prep_roberts_c2f(L, n, d, q)
        else:
            raise ValueError(f"bad distribution in mesh extend {caller} for mesh {dist}")
    return g


# ---- sub-domain overlap of two meshes ------------------------------------------

def _inside(p: float, lo: float, hi: float, tol: float) -> bool:
    """inside_OL: strictly inside, or within tol of either end."""
    return (lo < p < hi) or abs(p - lo) < tol or abs(p - hi) < tol


@dataclass
class Overlap:
    """Index ranges (1-based, inclusive, as the reference stores them) of the
    points two coordinate arrays share: i1 in the first, i2 in the second."""
    i1: Tuple[int, int]
    i2: Tuple[int, int]

    @property
    def iR(self) -> int:
        return self.i1[1] - self.i1[0] + 1

    @property
    def success(self) -> bool:
        return 0 not in (self.i1[0], self.i1[1], self.i2[0], self.i2[1])

    def valid_range(self) -> bool:
        return self.i1[1] - self.i1[0] == self.i2[1] - self.i2[0]


def _overlap_blind(h1, h2, n_cells1, n_cells2, tol, p) -> Overlap:
    i1 = [0, 0]
    i2 = [0, 0]
    p1 = p2 = p
    if p > 0:
        if n_cells1 == 1:
            p1 = 0
        if n_cells2 == 1:
            p2 = 0
    else:
        p1 = p2 = 0
    s1, s2 = len(h1), len(h2)
    for i in range(s1 - p1, p1, -1):
        for j in range(1 + p2, s2 - p2 + 1):
            if _inside(h2[j - 1], h1[i - 1], h1[i - 1], tol):
                i1[0] = i if i1[0] == 0 else min(i1[0], i)
                i1[1] = i if i1[1] == 0 else max(i1[1], i)
                i2[0] = j if i2[0] == 0 else min(i2[0], j)
                i2[1] = j if i2[1] == 0 else max(i2[1], j)
    return Overlap(tuple(i1), tuple(i2))


def n_overlap(hn1: np.ndarray, hn2: np.ndarray, tol: float = 1e-12, p: int = 1) -> Overlap:
    """get_N_overlap_OL: shared nodes; p = 1 skips the ghost node of each
    end (the physical overlap), p = 0 includes it (the total overlap)."""
    if p < 0:
        raise ValueError("bad input to get_N_overlap")
    sc1, sc2 = len(hn1) - 1, len(hn2) - 1
    if not (len(hn1) - p > 0 and len(hn2) - p > 0):
        p = 0
    return _overlap_blind(np.asarray(hn1), np.asarray(hn2), sc1, sc2, tol, p)


def c_overlap(hn1: np.ndarray, hn2: np.ndarray, tol: float = 1e-12, p: int = 1) -> Overlap:
    """get_C_overlap_OL: shared cell centres."""
    if p < 0:
        raise ValueError("bad input to get_C_overlap")
    hc1 = 0.5 * (np.asarray(hn1)[1:] + np.asarray(hn1)[:-1])
    hc2 = 0.5 * (np.asarray(hn2)[1:] + np.asarray(hn2)[:-1])
    if not (len(hc1) - p > 0 and len(hc2) - p > 0):
        p = 0
    return _overlap_blind(hc1, hc2, len(hc1), len(hc2), tol, p)


def is_overlap(hn1: np.ndarray, hn2: np.ndarray, tol: float = 1e-12) -> bool:
    """is_overlap_general over the full extents (amin, amax) of the two arrays."""
    a1, b1, a2, b2 = hn1[0], hn1[-1], hn2[0], hn2[-1]
    L = ((a1 > a2) and (a1 < b2), (b1 > a2) and (b1 < b2), abs(a2 - a1) < tol, abs(b2 - b1) < tol,
         (a1 > a2) and (b1 < b2), (a2 > a1) and (b2 < b1))
    return any(L)


def sub_domain_offset(inner: Sequence[np.ndarray], outer: Sequence[np.ndarray], tol: float = 1e-12) -> Tuple[int, int, int]:
    """Index shift of a mesh embedded in a larger one: per direction, the
    outer index of the inner mesh's first physical cell minus the inner
    index (the physical cell overlap of init_sub_domain with p = 1).  The
    inner physical cells must coincide with a contiguous run of outer cells."""
    off = []
    for d in range(3):
        if not is_overlap(inner[d], outer[d], tol):
            raise ValueError(f"meshes do not overlap along direction {d + 1}")
        ol = c_overlap(inner[d], outer[d], tol, 1)
        nphys = len(inner[d]) - 3
        if not ol.success or not ol.valid_range() or ol.iR != nphys:
            raise ValueError(f"the inner mesh's cells are not cells of the outer mesh along direction {d + 1}")
        off.append(ol.i2[0] - ol.i1[0])
    return tuple(off)


def sub_domain_ranges(inner: Sequence[np.ndarray], outer: Sequence[np.ndarray], tol: float = 1e-12):
    """Outer-mesh index ranges (0-based, end exclusive) of the inner mesh's
    physical cells and nodes per direction: ((c0, c1), (n0, n1)) each."""
    out = []
    for d in range(3):
        c = c_overlap(inner[d], outer[d], tol, 1)
        n = n_overlap(inner[d], outer[d], tol, 1)
        if not (c.success and n.success):
            raise ValueError(f"meshes do not overlap along direction {d + 1}")
        out.append(((c.i2[0] - 1, c.i2[1]), (n.i2[0] - 1, n.i2[1])))
    return out
