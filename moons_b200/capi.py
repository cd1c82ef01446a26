"""ctypes host mirror of the reference's field / operator / solver API.

The objects map one to one onto the reference's Fortran types and routines:

* ``Mesh``   -- a single-block mesh (HW/mesh, HW/grid coordinates)
* ``Field``  -- an SF with one block: data location, BCs, device array
* ``PCG``    -- PCG_solver_SF / PCG_solver_VF (HW/PCG/PCG_solver_extend.f90)
* ``grad/div/curl/lap_centered/lap_var/delta/interp`` -- HW/ops routines

Every call goes through the C-ABI of ``include/moons_gpu.h`` in
``moons_b200/lib/libmoons_gpu.so``; nothing here computes on the host.  A
missing library raises immediately -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from . import build as _build

CC, FX, FY, FZ, EX, EY, EZ, NODE = range(8)
DIRICHLET, NEUMANN, PERIODIC, ROBIN = 1, 2, 3, 4
OP_LAP_UNIFORM, OP_LAP_PROPS, OP_IND_DIFFUSION, OP_MOM_DIFFUSION, OP_NRG_DIFFUSION = 1, 2, 3, 4, 5
PREC_IDENTITY, PREC_LAP, PREC_MOM, PREC_IND = 0, 1, 2, 3
PREC_MG, PREC_MG_MIXED = 4, 5  # multigrid V-cycle in CG (FP64) / in flexible CG (FP32 V-cycle)
PREC_FD = 7  # direct solve of the separable Poisson operator (fast diagonalization) in CG
PREC_UNET_MG = 8  # learned + mixed: z = V(r) + N(r - A V(r)) in flexible CG (V the FP32 V-cycle)
PREC_UNET = 6  # learned U-Net in flexible CG, FP32 V-cycle fallback (PCG.set_unet)


class MoonsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"moons error {code}: {msg}")
        self.code = code


class BCSpec(C.Structure):
    _fields_ = [
        ("type", C.c_int * 6),
        ("prescribed", C.c_int * 6),
        ("value", C.c_double * 6),
        ("c_w", C.c_double * 6),
        ("order", C.c_int * 6),
        ("all_neumann", C.c_int),
    ]


class ISP(C.Structure):
    _fields_ = [
        ("iter_max", C.c_int),
        ("tol_rel", C.c_double),
        ("tol_abs", C.c_double),
        ("n_skip_check_res", C.c_int),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("res0", C.c_double),
        ("res", C.c_double),
        ("rel", C.c_double),
        ("exit_reason", C.c_int),
        ("ms", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


IND_OFF, IND_B, IND_POTENTIAL = 0, 1, 2
MHD_SIGMA_INV_CC, MHD_U_CC = 13, 14
MHD_U, MHD_P, MHD_B, MHD_B0, MHD_PHI, MHD_J, MHD_SIGMA_INV, MHD_JXB, MHD_DIVU, MHD_DIVB, MHD_T, MHD_KT, MHD_GRAVITY = \
    range(13)


class MHDParams(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("induction", C.c_int),
        ("finite_Rem", C.c_int),
        ("mpg_dir", C.c_int),
        ("mpg_scale", C.c_double),
        ("scale_advection_U", C.c_double),
        ("scale_diffusion_U", C.c_double),
        ("scale_JxB", C.c_double),
        ("scale_advection_B", C.c_double),
        ("scale_diffusion_B", C.c_double),
        ("scale_current", C.c_double),
        ("coeff_implicit_U", C.c_double),
        ("coeff_implicit_B", C.c_double),
        ("isp_U", ISP),
        ("isp_p", ISP),
        ("isp_B", ISP),
        ("isp_phi", ISP),
        ("bc_U", BCSpec * 3),
        ("bc_p", BCSpec),
        ("bc_B", BCSpec * 3),
        ("bc_phi", BCSpec),
        ("ind_offset", C.c_int * 3),
        ("prescribed_Ustar", C.c_int),
        ("prescribed_Bstar", C.c_int),
        ("prec_poisson", C.c_int),
        ("energy", C.c_int),
        ("solve_method_T", C.c_int),
        ("coeff_implicit_T", C.c_double),
        ("scale_advection_T", C.c_double),
        ("scale_diffusion_T", C.c_double),
        ("scale_heating_T", C.c_double),
        ("scale_buoyancy", C.c_double),
        ("isp_T", ISP),
        ("bc_T", BCSpec),
        ("scale_KE_diffusion_T", C.c_double),
        ("scale_viscous_dissipation_T", C.c_double),
        ("scale_joule_heating_T", C.c_double),
        ("solve_method_U", C.c_int),
        ("solve_method_B", C.c_int),
        ("rk_stages", C.c_int),
        ("scale_diffusion_linear_U", C.c_double),
        ("scale_diffusion_linear_B", C.c_double),
    ]


class StepInfo(C.Structure):
    _fields_ = [
        ("steps", C.c_int),
        ("iters_U", C.c_int),
        ("iters_p", C.c_int),
        ("iters_B", C.c_int),
        ("iters_phi", C.c_int),
        ("res_p", C.c_double),
        ("res_phi", C.c_double),
        ("ms", C.c_double),
        ("iters_T", C.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def bc_spec(types: Sequence[int], values: Sequence[float] | None = None,
            prescribed: Sequence[int] | None = None, c_w: Sequence[float] | None = None,
            order: Sequence[int] | None = None, all_neumann: bool = False) -> BCSpec:
    s = BCSpec()
    for f in range(6):
        s.type[f] = int(types[f])
        s.value[f] = float(values[f]) if values is not None else 0.0
        s.prescribed[f] = int(prescribed[f]) if prescribed is not None else 0
        s.c_w[f] = float(c_w[f]) if c_w is not None else 0.0
        s.order[f] = int(order[f]) if order is not None else f + 1
    s.all_neumann = 1 if all_neumann else 0
    return s


def isp(iter_max: int, tol_rel: float, tol_abs: float, n_skip_check_res: int = 1) -> ISP:
    return ISP(int(iter_max), float(tol_rel), float(tol_abs), int(n_skip_check_res))


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)


class _Lib:
    """Loads a shared library exposing the MOONS entry points under ``prefix``."""

    def __init__(self, path: str, prefix: str):
        self.path = path
        self.lib = C.CDLL(path)
        self.prefix = prefix

    def fn(self, name, restype, argtypes):
        f = getattr(self.lib, self.prefix + name)
        f.restype = restype
        f.argtypes = argtypes
        return f


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            raise RuntimeError(f"MOONS CUDA library missing: {path} (run python -m moons_b200.build)")
        L = C.CDLL(path)
        sig = {
            "moons_last_error": (C.c_char_p, []),
            "moons_mesh_create": (C.c_int, [C.POINTER(_P), _D, C.c_int, _D, C.c_int, _D, C.c_int, C.c_int]),
            "moons_mesh_destroy": (C.c_int, [_P]),
            "moons_mesh_sync": (C.c_int, [_P]),
            "moons_sf_create": (C.c_int, [_P, C.c_int, C.POINTER(_P)]),
            "moons_sf_destroy": (C.c_int, [_P]),
            "moons_sf_shape": (C.c_int, [_P, C.POINTER(C.c_int)]),
            "moons_sf_upload": (C.c_int, [_P, _D, C.c_longlong]),
            "moons_sf_download": (C.c_int, [_P, _D, C.c_longlong]),
            "moons_sf_fill": (C.c_int, [_P, C.c_double]),
            "moons_sf_set_bcs": (C.c_int, [_P, C.POINTER(BCSpec)]),
            "moons_apply_bcs": (C.c_int, [_P]),
            "moons_apply_bcs_implicit": (C.c_int, [_P]),
            "moons_del": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int]),
            "moons_grad": (C.c_int, [_P, _P, _P, _P]),
            "moons_div": (C.c_int, [_P, _P, _P, _P]),
            "moons_curl": (C.c_int, [_P, _P, _P, _P, _P, _P]),
            "moons_lap_centered": (C.c_int, [_P, _P]),
            "moons_lap_var": (C.c_int, [_P, _P, _P, _P, _P]),
            "moons_lap_var_noalloc": (C.c_int, [_P, _P, _P, _P, _P]),
            "moons_interp": (C.c_int, [_P, _P, C.c_int]),
            "moons_pcg_create": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.POINTER(_P), C.POINTER(_P),
                                           C.POINTER(_P), C.POINTER(_P)]),
            "moons_pcg_destroy": (C.c_int, [_P]),
            "moons_pcg_update_mfp": (C.c_int, [_P, C.c_double, C.c_int]),
            "moons_pcg_solve": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(ISP), C.POINTER(SolveInfo)]),
            "moons_mhd_create": (C.c_int, [_P, _P, C.POINTER(MHDParams), C.POINTER(_P)]),
            "moons_mhd_destroy": (C.c_int, [_P]),
            "moons_mhd_field": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(_P)]),
            "moons_mhd_init": (C.c_int, [_P]),
            "moons_mhd_set_unet": (C.c_int, [_P, C.c_int, _P]),
            "moons_mhd_step": (C.c_int, [_P, C.c_int, C.POINTER(StepInfo)]),
            "moons_mhd_divergence": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
            "moons_kernel_launches": (C.c_longlong, []),
            "moons_debug_bounded_wait": (C.c_int, [C.c_ulonglong]),
            "moons_mg_level_shape": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "moons_mg_debug": (C.c_int, [_P, C.c_int, C.c_int, _D, _D, _D]),
            "moons_unet_create": (C.c_int, [_P, C.c_ulonglong, C.POINTER(_P)]),
            "moons_unet_destroy": (C.c_int, [_P]),
            "moons_unet_nparams": (C.c_int, [_P, C.POINTER(C.c_longlong)]),
            "moons_unet_get_params": (C.c_int, [_P, _F, C.c_longlong]),
            "moons_unet_set_params": (C.c_int, [_P, _F, C.c_longlong]),
            "moons_unet_set_out_scale": (C.c_int, [_P, C.c_double]),
            "moons_unet_get_out_scale": (C.c_int, [_P, C.POINTER(C.c_double)]),
            "moons_unet_set_feature": (C.c_int, [_P, _F, C.c_longlong]),
            "moons_unet_apply": (C.c_int, [_P, _P, _P]),
            "moons_unet_set_coeff": (C.c_int, [_P, _P, _P, _P]),
            "moons_unet_set_loss": (C.c_int, [_P, C.c_int]),
            "moons_unet_set_operator": (C.c_int, [_P, _P]),
            "moons_pcg_set_unet": (C.c_int, [_P, _P]),
            "moons_pcg_residual": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
            "moons_pcg_apply_prec": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P)]),
            "moons_pcg_apply_op": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P)]),
            "moons_clean_div": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), _P, C.c_double, C.POINTER(_P), _P,
                                          C.POINTER(ISP), C.POINTER(SolveInfo)]),
            "moons_unet_loss_grad": (C.c_int, [_P, _P, _P, _F, _F, C.c_longlong]),
            "moons_unet_train_step": (C.c_int, [_P, _P, _P, C.c_float, _F]),
            "moons_unet_layer_check": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                                 _F, _F, _F, _F, C.c_int, _F]),
        }
        for name, (rt, at) in sig.items():
            f = getattr(L, name)
            f.restype = rt
            f.argtypes = at
        _lib = L
    return _lib


def _check(code: int):
    if code != 0:
        raise MoonsError(code, lib().moons_last_error().decode())


def _arr(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_D)


class Mesh:
    def __init__(self, hx, hy, hz, device: int = -1):
        L = lib()
        self._keep = [_arr(h)[0] for h in (hx, hy, hz)]
        h = _P()
        _check(L.moons_mesh_create(C.byref(h), self._keep[0].ctypes.data_as(_D), len(self._keep[0]),
                                   self._keep[1].ctypes.data_as(_D), len(self._keep[1]),
                                   self._keep[2].ctypes.data_as(_D), len(self._keep[2]), device))
        self.h = h
        self.sn = tuple(len(k) for k in self._keep)

    def field(self, dl: int) -> "Field":
        return Field(self, dl)

    def sync(self):
        _check(lib().moons_mesh_sync(self.h))

    def close(self):
        if self.h:
            lib().moons_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Field:
    def __init__(self, mesh: Mesh, dl: int):
        self.mesh = mesh
        self.dl = dl
        h = _P()
        _check(lib().moons_sf_create(mesh.h, dl, C.byref(h)))
        self.h = h
        s = (C.c_int * 3)()
        _check(lib().moons_sf_shape(h, s))
        self.shape = (s[0], s[1], s[2])

    @property
    def n(self):
        return self.shape[0] * self.shape[1] * self.shape[2]

    def upload(self, a: np.ndarray):
        a = np.asarray(a, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"shape {a.shape} != field {self.shape}")
        flat = np.ascontiguousarray(a.ravel(order="F"))
        _check(lib().moons_sf_upload(self.h, flat.ctypes.data_as(_D), flat.size))

    def download(self) -> np.ndarray:
        flat = np.empty(self.n, dtype=np.float64)
        _check(lib().moons_sf_download(self.h, flat.ctypes.data_as(_D), flat.size))
        return flat.reshape(self.shape, order="F")

    def fill(self, v: float):
        _check(lib().moons_sf_fill(self.h, float(v)))

    def set_bcs(self, spec: BCSpec):
        _check(lib().moons_sf_set_bcs(self.h, C.byref(spec)))

    def apply_bcs(self):
        _check(lib().moons_apply_bcs(self.h))

    def apply_bcs_implicit(self):
        _check(lib().moons_apply_bcs_implicit(self.h))

    def close(self):
        if self.h:
            lib().moons_sf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def delta(out: Field, inp: Field, n: int, d: int, pad: int, gen: int):
    _check(lib().moons_del(out.h, inp.h, n, d, pad, gen))


def grad(gx: Field, gy: Field, gz: Field, u: Field):
    _check(lib().moons_grad(gx.h, gy.h, gz.h, u.h))


def div(o: Field, ux: Field, uy: Field, uz: Field):
    _check(lib().moons_div(o.h, ux.h, uy.h, uz.h))


def curl(o: Sequence[Field], u: Sequence[Field]):
    _check(lib().moons_curl(o[0].h, o[1].h, o[2].h, u[0].h, u[1].h, u[2].h))


def lap_centered(o: Field, u: Field):
    _check(lib().moons_lap_centered(o.h, u.h))


def lap_var(o: Field, u: Field, k: Sequence[Field]):
    _check(lib().moons_lap_var(o.h, u.h, k[0].h, k[1].h, k[2].h))


def lap_var_noalloc(o: Field, u: Field, k: Sequence[Field]):
    """lap_var without device allocation: the face temporaries come from a
    built-in device array (at most LAP_VAR_NOALLOC_MAX_POINTS points each;
    larger fields raise MoonsError with MOONS_ERR_LIMIT).  Calls that overlap
    in time race on that array."""
    _check(lib().moons_lap_var_noalloc(o.h, u.h, k[0].h, k[1].h, k[2].h))


LAP_VAR_NOALLOC_MAX_POINTS = 131072


def interp(o: Field, i: Field, d: int):
    _check(lib().moons_interp(o.h, i.h, d))


def _ptrs(fs):
    arr = (_P * 3)()
    for i, f in enumerate(fs):
        arr[i] = f.h if f is not None else None
    return arr


class _FieldView:
    """A field owned by an MHD object (upload/download/shape only)."""

    def __init__(self, owner, h):
        self.owner = owner
        self.h = h
        s = (C.c_int * 3)()
        _check(lib().moons_sf_shape(h, s))
        self.shape = (s[0], s[1], s[2])

    @property
    def n(self):
        return self.shape[0] * self.shape[1] * self.shape[2]

    upload = Field.upload
    download = Field.download

    def upload_ptr(self, ptr: int):
        """Copy n doubles from host address ``ptr`` (e.g. pinned memory)."""
        _check(lib().moons_sf_upload(self.h, C.cast(ptr, _D), self.n))

    def download_ptr(self, ptr: int):
        _check(lib().moons_sf_download(self.h, C.cast(ptr, _D), self.n))


def clean_div(pcg: "PCG", X, Xstar, phi, scale: float, temp_F, temp_CC, params) -> dict:
    """clean_div (clean_divergence.f90:37-59): project Xstar onto X with the
    potential phi solved by `pcg` (LAP_UNIFORM on phi's layout)."""
    info = SolveInfo()
    _check(lib().moons_clean_div(pcg.h, _ptrs(X), _ptrs(Xstar), phi.h, float(scale), _ptrs(temp_F), temp_CC.h,
                                 C.byref(params), C.byref(info)))
    return info.as_dict()


class MHD:
    """The MHD time-step object (solve_MOONS for one block pair)."""

    def __init__(self, mesh_mom: Mesh, mesh_ind: Mesh, params: MHDParams):
        self.meshes = (mesh_mom, mesh_ind)
        self.params = params
        h = _P()
        _check(lib().moons_mhd_create(mesh_mom.h, mesh_ind.h, C.byref(params), C.byref(h)))
        self.h = h

    def field(self, which: int, comp: int = 0):
        f = _P()
        _check(lib().moons_mhd_field(self.h, which, comp, C.byref(f)))
        return _FieldView(self, f)

    def upload(self, which, comp, a):
        self.field(which, comp).upload(a)

    def download(self, which, comp=0):
        return self.field(which, comp).download()

    def shape(self, which, comp=0):
        return self.field(which, comp).shape

    def init(self):
        _check(lib().moons_mhd_init(self.h))

    def set_unet(self, which: int, net: "UNet"):
        """Network of the learned + mixed pressure (0) or B-form cleaning
        potential (1) solve (prec_poisson = PREC_UNET_MG); kept alive here."""
        _check(lib().moons_mhd_set_unet(self.h, int(which), net.h))
        if not hasattr(self, "nets"):
            self.nets = {}
        self.nets[which] = net

    def step(self, n: int = 1) -> dict:
        info = StepInfo()
        _check(lib().moons_mhd_step(self.h, int(n), C.byref(info)))
        return info.as_dict()

    def divergence(self):
        a, b = C.c_double(), C.c_double()
        _check(lib().moons_mhd_divergence(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def close(self):
        if self.h:
            lib().moons_mhd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PCG:
    """PCG_solver_SF (ncomp=1) / PCG_solver_VF (ncomp=3)."""

    def __init__(self, mesh: Mesh, op: int, prec: int, x: Sequence[Field], x_bc: Sequence[Field],
                 k: Sequence[Field] | None = None):
        self.mesh = mesh
        self.nc = len(x)
        h = _P()
        _check(lib().moons_pcg_create(mesh.h, op, prec, self.nc, _ptrs(x), _ptrs(x_bc),
                                      _ptrs(k) if k is not None else None, C.byref(h)))
        self.h = h

    def update_mfp(self, coeff: float, update_prec: bool = True):
        _check(lib().moons_pcg_update_mfp(self.h, float(coeff), 1 if update_prec else 0))

    def mg_level_shape(self, level: int):
        """(extents of the level's cell-centred arrays, number of levels) of an
        MOONS_PREC_MG solver's hierarchy."""
        s = (C.c_int * 3)()
        nl = C.c_int()
        _check(lib().moons_mg_level_shape(self.h, int(level), s, C.byref(nl)))
        return (s[0], s[1], s[2]), nl.value

    def mg_debug(self, op: int, level: int, a, b=None):
        """One multigrid building block on host arrays (moons_mg_debug): op 0
        prolongation (a on level+1), 1 restriction (result on level+1), 2 a
        red and a black SOR sweep, 3 the residual b - A a."""
        out_level = level + 1 if op == 1 else level
        shp, _ = self.mg_level_shape(out_level)
        aa = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
        bb = None if b is None else np.ascontiguousarray(np.asarray(b, dtype=np.float64).ravel(order="F"))
        out = np.zeros(shp[0] * shp[1] * shp[2])
        _check(lib().moons_mg_debug(self.h, int(op), int(level), aa.ctypes.data_as(_D),
                                    None if bb is None else bb.ctypes.data_as(_D), out.ctypes.data_as(_D)))
        return out.reshape(shp, order="F")

    def residual(self, x: Sequence[Field], b: Sequence[Field], out: Sequence[Field]):
        """The solver's internal residual vol*(b - A x) for the iterate x."""
        _check(lib().moons_pcg_residual(self.h, _ptrs(x), _ptrs(b), _ptrs(out)))

    def apply_op(self, out: Sequence[Field], x: Sequence[Field]):
        """out = A x with the solver's operator (operator_explicit form)."""
        _check(lib().moons_pcg_apply_op(self.h, _ptrs(out), _ptrs(x)))

    def apply_prec(self, z: Sequence[Field], r: Sequence[Field]):
        """z = M(r) with the solver's preconditioner (a multigrid-family
        solver applies one V-cycle alone)."""
        _check(lib().moons_pcg_apply_prec(self.h, _ptrs(z), _ptrs(r)))

    def set_unet(self, net: "UNet"):
        """Attach the network of a PREC_UNET / PREC_UNET_MG solver (kept alive
        by the solver)."""
        _check(lib().moons_pcg_set_unet(self.h, net.h))
        self.net = net

    def solve(self, x: Sequence[Field], b: Sequence[Field], params: ISP) -> dict:
        info = SolveInfo()
        _check(lib().moons_pcg_solve(self.h, _ptrs(x), _ptrs(b), C.byref(params), C.byref(info)))
        return info.as_dict()

    def close(self):
        if self.h:
            lib().moons_pcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def debug_bounded_wait(limit_ns: int):
    """Run one bounded in-kernel wait that nothing completes (raises
    MoonsError MOONS_ERR_CUDA naming the site once the limit has passed)."""
    _check(lib().moons_debug_bounded_wait(int(limit_ns)))


def kernel_launches() -> int:
    """Kernels this process launched through the library (host launches plus
    the launches executed inside the solver's device-side loop)."""
    return int(lib().moons_kernel_launches())


def _fp(a):
    return None if a is None else a.ctypes.data_as(_F)


class UNet:
    """The learned preconditioner (3-D U-Net) on a mesh's cell-centred
    interior; see moons_unet_* in include/moons_gpu.h."""

    def __init__(self, mesh: Mesh, seed: int = 0):
        self.mesh = mesh
        h = _P()
        _check(lib().moons_unet_create(mesh.h, int(seed), C.byref(h)))
        self.h = h
        n = C.c_longlong()
        _check(lib().moons_unet_nparams(h, C.byref(n)))
        self.nparams = int(n.value)

    def get_params(self) -> np.ndarray:
        a = np.empty(self.nparams, dtype=np.float32)
        _check(lib().moons_unet_get_params(self.h, _fp(a), self.nparams))
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        _check(lib().moons_unet_set_params(self.h, _fp(a), a.size))

    @property
    def out_scale(self) -> float:
        c = C.c_double()
        _check(lib().moons_unet_get_out_scale(self.h, C.byref(c)))
        return c.value

    @out_scale.setter
    def out_scale(self, c: float):
        _check(lib().moons_unet_set_out_scale(self.h, float(c)))

    def set_feature(self, feat):
        a = np.ascontiguousarray(np.asarray(feat, dtype=np.float32).ravel(order="F"))
        _check(lib().moons_unet_set_feature(self.h, _fp(a), a.size))

    def set_loss(self, kind: int):
        """Training loss: 0 relative L2, 1 cosine (scale-invariant, default),
        2 cosine in the energy norm of the operator set by set_operator."""
        _check(lib().moons_unet_set_loss(self.h, int(kind)))

    def set_operator(self, solver: "PCG"):
        """The operator of the energy-norm loss (an MG_MIXED / UNET solver)."""
        _check(lib().moons_unet_set_operator(self.h, solver.h))

    def set_coeff(self, k: Sequence[Field]):
        """Feature from the face coefficients of a LAP_PROPS operator."""
        _check(lib().moons_unet_set_coeff(self.h, k[0].h, k[1].h, k[2].h))

    def apply(self, z: Field, r: Field):
        _check(lib().moons_unet_apply(self.h, z.h, r.h))

    def loss_grad(self, r: Field, e: Field, want_grads: bool = True):
        loss = np.zeros(1, dtype=np.float32)
        g = np.empty(self.nparams, dtype=np.float32) if want_grads else None
        _check(lib().moons_unet_loss_grad(self.h, r.h, e.h, _fp(loss), _fp(g), self.nparams if want_grads else 0))
        return float(loss[0]), g

    def train_step(self, r: Field, e: Field, lr: float) -> float:
        loss = np.zeros(1, dtype=np.float32)
        _check(lib().moons_unet_train_step(self.h, r.h, e.h, float(lr), _fp(loss)))
        return float(loss[0])

    def close(self):
        if self.h:
            lib().moons_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def unet_layer_check(op: int, X: int, Y: int, Z: int, cinA: int, cinB: int, cout: int, inp=None, dout=None,
                     W=None, bias=None, relu: bool = True) -> np.ndarray:
    """Run one U-Net layer kernel on host data (see moons_unet_layer_check)."""
    cin = cinA + cinB
    f32 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)
    inp, dout, W, bias = f32(inp), f32(dout), f32(W), f32(bias)
    n = {0: cout * X * Y * Z, 1: cin * X * Y * Z, 2: cout * cin * 27 + cout}[op]
    out = np.empty(n, dtype=np.float32)
    _check(lib().moons_unet_layer_check(op, X, Y, Z, cinA, cinB, cout, _fp(inp), _fp(dout), _fp(W), _fp(bias),
                                        int(relu), _fp(out)))
    return out
