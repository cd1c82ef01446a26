"""The reference's mesh bank (code/handwritten/sim_params/mesh_bank.f90).

Each preset returns the segment lists of the three meshes of a case:
``mom`` (the fluid), ``sigma`` (fluid plus conducting walls) and ``ind``
(the induction mesh: the conductor plus any vacuum around it).  As in the
reference, ``sigma`` starts as a copy of ``mom`` and ``ind`` as a copy of
``sigma`` (or the other way round where a preset says so), each with its
own extensions added.  The cell counts default to the reference's values
and can be lowered for tests; ``mqp`` defaults to the setting every
sim_params_init_mesh of the reference uses, init(MQP, T, 2.0, 50).

``generate`` turns a preset into node coordinates (with ghost nodes) for
the given Reynolds and Hartmann numbers (generate_mesh_generic).
"""
from __future__ import annotations

import math
from typing import NamedTuple, Tuple

import numpy as np

from .mesh_gen import Grid, MeshParams, MeshQuality, generate_mesh_generic, seg_1d

PI = 3.141592653589793238462643383279502884197169399375105820974


def default_quality() -> MeshQuality:
    return MeshQuality(True, 2.0, 50)


class MeshSet(NamedTuple):
    mom: MeshParams
    sigma: MeshParams
    ind: MeshParams


class Meshes(NamedTuple):
    mom: Tuple[np.ndarray, np.ndarray, np.ndarray]
    sigma: Tuple[np.ndarray, np.ndarray, np.ndarray]
    ind: Tuple[np.ndarray, np.ndarray, np.ndarray]


def generate(ms: MeshSet, Re: float, Ha: float) -> Meshes:
    return Meshes(*(generate_mesh_generic(mp, Re, Ha, name).coords()
                    for mp, name in ((ms.mom, "mom"), (ms.sigma, "sigma"), (ms.ind, "ind"))))


def _new(mqp):
    q = mqp if mqp is not None else default_quality()
    return MeshParams(q), q


def plasma_disruption(N=100, N_w=14, mqp=None) -> MeshSet:
    """define_mesh_SP_plasma_disruption (mesh_bank.f90:33-52)."""
    CR, t_fluid, t_wall, buffer = 10.0, 1.0, 0.05, 1.5
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_Roberts_B", N * 2, -t_fluid * CR, t_fluid * CR, buffer))
    mom.add_base(seg_1d(2, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    mom.add_base(seg_1d(3, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    sigma = mom.copy()
    sigma.add_ext(seg_1d(1, "ext_Roberts_B_IO", N_w * 2, t_wall, buffer))
    sigma.add_ext(seg_1d(2, "ext_Roberts_B_IO", N_w, t_wall, buffer))
    sigma.add_ext(seg_1d(3, "ext_Roberts_B_IO", N_w, t_wall, buffer))
    return MeshSet(mom, sigma, sigma.copy())


def plasma_disruption_plane(N=130, N_w=14, mqp=None) -> MeshSet:
    """define_mesh_SP_plasma_disruption_plane (mesh_bank.f90:54-71)."""
    t_fluid, t_wall, buffer = 1.0, 0.05, 1.5
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", 1, -0.5, 0.5, buffer))
    mom.add_base(seg_1d(2, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    mom.add_base(seg_1d(3, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    sigma = mom.copy()
    sigma.add_ext(seg_1d(2, "ext_Roberts_B_IO", N_w, t_wall, buffer))
    sigma.add_ext(seg_1d(3, "ext_Roberts_B_IO", N_w, t_wall, buffer))
    return MeshSet(mom, sigma, sigma.copy())


def plasma_disruption_plane_insulating(N=150, mqp=None) -> MeshSet:
    """define_mesh_SP_plasma_disruption_plane_insulating (mesh_bank.f90:73-88)."""
    t_fluid, buffer = 1.0, 1.5
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", 1, -0.5, 0.5, buffer))
    mom.add_base(seg_1d(2, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    mom.add_base(seg_1d(3, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    sigma = mom.copy()
    return MeshSet(mom, sigma, sigma.copy())


def plasma_disruption_line(N=200, N_w=14, mqp=None) -> MeshSet:
    """define_mesh_SP_plasma_disruption_line (mesh_bank.f90:90-106)."""
    t_fluid, t_wall, buffer = 1.0, 0.05, 1.5
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", 1, -0.5, 0.5, buffer))
    mom.add_base(seg_1d(2, "grid_uniform", 1, -0.5, 0.5, buffer))
    mom.add_base(seg_1d(3, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    sigma = mom.copy()
    sigma.add_ext(seg_1d(3, "ext_Roberts_B_IO", N_w, t_wall, buffer))
    return MeshSet(mom, sigma, sigma.copy())


def plasma_disruption_1d_analytic(N=100, mqp=None) -> MeshSet:
    """define_mesh_SP_plasma_disruption_1D_analytic (mesh_bank.f90:108-122)."""
    t_fluid, buffer = 1.0, 1.5
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", 1, -t_fluid, t_fluid, buffer))
    mom.add_base(seg_1d(2, "grid_uniform", 1, -t_fluid, t_fluid, buffer))
    mom.add_base(seg_1d(3, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    sigma = mom.copy()
    return MeshSet(mom, sigma, sigma.copy())


def small_dataset(N=5, mqp=None) -> MeshSet:
    """small_dataset (mesh_bank.f90:124-137)."""
    t_fluid, buffer = 1.0, 1.0
    mom, q = _new(mqp)
    for d in (1, 2, 3):
        mom.add_base(seg_1d(d, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    sigma = mom.copy()
    return MeshSet(mom, sigma, sigma.copy())


def bandaru(N=130, mqp=None) -> MeshSet:
    """define_mesh_bandaru (mesh_bank.f90:139-152): ind copies mom, sigma copies ind."""
    buffer = 1.0
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", N, 0.0, 2.0 * PI, buffer))
    mom.add_base(seg_1d(3, "grid_Roberts_B", N, -1.0, 1.0, buffer))
    mom.add_base(seg_1d(2, "grid_uniform", 1, -0.5, 0.5, buffer))
    ind = mom.copy()
    return MeshSet(mom, ind.copy(), ind)


def bandaru_fft(N=128, mqp=None) -> MeshSet:
    """define_mesh_bandaru_FFT (mesh_bank.f90:154-167)."""
    buffer = 1.0
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", N, 0.0, 2.0 * PI, buffer))
    mom.add_base(seg_1d(3, "grid_uniform", N * 2, -1.0, 1.0, buffer))
    mom.add_base(seg_1d(2, "grid_uniform", 1, -0.5, 0.5, buffer))
    ind = mom.copy()
    return MeshSet(mom, ind.copy(), ind)


def mhd_shercliff_plane(N=150, mqp=None) -> MeshSet:
    """define_mesh_MHD_Shercliff_plane (mesh_bank.f90:169-182)."""
    buffer = 1.0
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", 1, -0.5, 0.5, buffer))
    mom.add_base(seg_1d(2, "grid_Roberts_B", N, -1.0, 1.0, buffer))
    mom.add_base(seg_1d(3, "grid_Roberts_B", N, -1.0, 1.0, buffer))
    ind = mom.copy()
    return MeshSet(mom, ind.copy(), ind)


def mhd_shercliff_plane_fft(N=128, mqp=None) -> MeshSet:
    """define_mesh_MHD_Shercliff_plane_FFT (mesh_bank.f90:184-197)."""
    buffer = 1.0
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", 1, -0.5, 0.5, buffer))
    mom.add_base(seg_1d(2, "grid_uniform", N, -0.5, 0.5, buffer))
    mom.add_base(seg_1d(3, "grid_uniform", N, -0.5, 0.5, buffer))
    ind = mom.copy()
    return MeshSet(mom, ind.copy(), ind)


def _full_bc_fluid(mom, N, N_half, t_fluid, buffer, roberts_b_z):
    mom.add_base(seg_1d(1, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    if roberts_b_z:
        mom.add_base(seg_1d(3, "grid_Roberts_B", N, -t_fluid, t_fluid, buffer))
    else:
        mom.add_base(seg_1d(3, "grid_Roberts_L", N_half, -t_fluid, 0.0, buffer))
    mom.add_base(seg_1d(2, "grid_Roberts_R", N_half + 5, 0.0, t_fluid, buffer))
    mom.add_ext(seg_1d(2, "ext_prep_Roberts_C2F_IO", N_half, 0.0 + t_fluid, buffer))


def full_bc_w_vacuum_symmetric(N=80, N_w=9, mqp=None) -> MeshSet:
    """define_mesh_full_BC_w_vacuum_symmetric (mesh_bank.f90:199-220):
    fluid clustered at its walls, a thin conducting wall (sigma), a vacuum
    region out to t_vac (ind); half domain in z."""
    t_vac, t_fluid, t_wall, buffer = 7.0, 1.0, 0.05, 2.0
    N_half = math.ceil(N / 2.0)
    mom, q = _new(mqp)
    _full_bc_fluid(mom, N, N_half, t_fluid, buffer, False)
    sigma = mom.copy()
    sigma.add_ext(seg_1d(1, "ext_Roberts_B_IO", N_w - 1, t_wall, buffer))
    sigma.add_ext(seg_1d(3, "ext_prep_Roberts_B_IO", N_w - 1, t_wall, buffer))
    sigma.add_ext(seg_1d(2, "ext_prep_Roberts_B_IO", N_w - 1, t_wall, buffer))
    ind = sigma.copy()
    ind.add_ext(seg_1d(1, "ext_Roberts_near_IO", N_w + 1, t_vac - t_fluid - t_wall, buffer))
    ind.add_ext(seg_1d(3, "ext_prep_Roberts_R_IO", N_w + 2, t_vac - t_fluid - t_wall, buffer))
    ind.add_ext(seg_1d(2, "ext_prep_Roberts_R_IO", N_w - 1, t_vac - t_fluid - t_wall, buffer))
    ind.add_ext(seg_1d(2, "ext_app_Roberts_L_IO", 2 * N_w - 2, t_vac - t_fluid, buffer))
    return MeshSet(mom, sigma, ind)


def full_bc_n_vacuum_symmetric(N=80, N_w=9, mqp=None) -> MeshSet:
    """define_mesh_full_BC_n_vacuum_symmetric (mesh_bank.f90:222-240): no vacuum."""
    t_fluid, t_wall, buffer = 1.0, 0.05, 2.0
    N_half = math.ceil(N / 2.0)
    mom, q = _new(mqp)
    _full_bc_fluid(mom, N, N_half, t_fluid, buffer, False)
    sigma = mom.copy()
    sigma.add_ext(seg_1d(1, "ext_Roberts_B_IO", N_w - 1, t_wall, buffer))
    sigma.add_ext(seg_1d(3, "ext_prep_Roberts_B_IO", N_w - 1, t_wall, buffer))
    sigma.add_ext(seg_1d(2, "ext_prep_Roberts_B_IO", N_w - 1, t_wall, buffer))
    return MeshSet(mom, sigma, sigma.copy())


def full_bc_w_vacuum_3d(N=80, N_w=9, mqp=None) -> MeshSet:
    """define_mesh_full_BC_w_vacuum_3D (mesh_bank.f90:242-265), the mesh of
    the reference's full_BC case: walls on five sides, the lid side open,
    vacuum all round."""
    t_vac, t_fluid, t_wall, buffer = 7.0, 1.0, 0.05, 2.0
    N_half = math.ceil(N / 2.0)
    mom, q = _new(mqp)
    _full_bc_fluid(mom, N, N_half, t_fluid, buffer, True)
    sigma = mom.copy()
    sigma.add_ext(seg_1d(1, "ext_Roberts_B_IO", N_w - 1, t_wall, buffer))
    sigma.add_ext(seg_1d(3, "ext_Roberts_B_IO", N_w - 1, t_wall, buffer))
    sigma.add_ext(seg_1d(2, "ext_prep_Roberts_B_IO", N_w - 1, t_wall, buffer))
    ind = sigma.copy()
    ind.add_ext(seg_1d(1, "ext_Roberts_near_IO", N_w + 1, t_vac - t_fluid - t_wall, buffer))
    ind.add_ext(seg_1d(3, "ext_Roberts_near_IO", N_w + 1, t_vac - t_fluid - t_wall, buffer))
    ind.add_ext(seg_1d(2, "ext_prep_Roberts_R_IO", N_w - 1, t_vac - t_fluid - t_wall, buffer))
    ind.add_ext(seg_1d(2, "ext_app_Roberts_L_IO", 2 * N_w - 2, t_vac - t_fluid, buffer))
    return MeshSet(mom, sigma, ind)


def full_bc_w_vacuum_3d_high_res(N=100, N_w=9, mqp=None) -> MeshSet:
    """define_mesh_full_BC_w_vacuum_3D_high_res (mesh_bank.f90:267-290)."""
    return full_bc_w_vacuum_3d(N, N_w, mqp)


def full_bc_n_vacuum_3d(N=80, N_w=9, mqp=None) -> MeshSet:
    """define_mesh_full_BC_n_vacuum_3D (mesh_bank.f90:292-310)."""
    t_fluid, t_wall, buffer = 1.0, 0.05, 2.0
    N_half = math.ceil(N / 2.0)
    mom, q = _new(mqp)
    _full_bc_fluid(mom, N, N_half, t_fluid, buffer, True)
    sigma = mom.copy()
    sigma.add_ext(seg_1d(1, "ext_Roberts_B_IO", N_w - 1, t_wall, buffer))
    sigma.add_ext(seg_1d(3, "ext_Roberts_B_IO", N_w - 1, t_wall, buffer))
    sigma.add_ext(seg_1d(2, "ext_prep_Roberts_B_IO", N_w - 1, t_wall, buffer))
    return MeshSet(mom, sigma, sigma.copy())


def mhd_ldc_sergey_uniform(N=45, N_ext=11, mqp=None) -> MeshSet:
    """define_mesh_SP_MHD_LDC_Sergey_uniform (mesh_bank.f90:312-326):
    uniform cavity, the induction mesh extended uniformly by N_ext cells on
    every side; sigma copies ind before the extension."""
    mom, q = _new(mqp)
    for d in (1, 2, 3):
        mom.add_base(seg_1d(d, "grid_uniform", N, -1.0, 1.0, 1.0))
    ind = mom.copy()
    sigma = ind.copy()
    for d in (1, 2, 3):
        ind.add_ext(seg_1d(d, "ext_uniform_IO", N_ext))
    return MeshSet(mom, sigma, ind)


def hydro_ldc_ghia(N=64, mqp=None) -> MeshSet:
    """define_mesh_hydro_LDC_Ghia (mesh_bank.f90:328-341): 2-D cavity, one cell in z."""
    buffer = 1.0
    mom, q = _new(mqp)
    mom.add_base(seg_1d(1, "grid_uniform", N, -1.0, 1.0, buffer))
    mom.add_base(seg_1d(2, "grid_uniform", N, -1.0, 1.0, buffer))
    mom.add_base(seg_1d(3, "grid_uniform", 1, -0.5, 0.5, buffer))
    ind = mom.copy()
    return MeshSet(mom, ind.copy(), ind)


PRESETS = {
    "plasma_disruption": plasma_disruption,
    "plasma_disruption_plane": plasma_disruption_plane,
    "plasma_disruption_plane_insulating": plasma_disruption_plane_insulating,
    "plasma_disruption_line": plasma_disruption_line,
    "plasma_disruption_1d_analytic": plasma_disruption_1d_analytic,
    "small_dataset": small_dataset,
    "bandaru": bandaru,
    "bandaru_fft": bandaru_fft,
    "mhd_shercliff_plane": mhd_shercliff_plane,
    "mhd_shercliff_plane_fft": mhd_shercliff_plane_fft,
    "full_bc_w_vacuum_symmetric": full_bc_w_vacuum_symmetric,
    "full_bc_n_vacuum_symmetric": full_bc_n_vacuum_symmetric,
    "full_bc_w_vacuum_3d": full_bc_w_vacuum_3d,
    "full_bc_w_vacuum_3d_high_res": full_bc_w_vacuum_3d_high_res,
    "full_bc_n_vacuum_3d": full_bc_n_vacuum_3d,
    "mhd_ldc_sergey_uniform": mhd_ldc_sergey_uniform,
    "hydro_ldc_ghia": hydro_ldc_ghia,
}
