"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Exposes the same Python surface as ``moons_b200.capi`` (Mesh, Field, grad,
div, curl, lap_centered, lap_var, delta, interp, PCG) but backed by the C++
restatement in ``oracle/moons_oracle.cpp``.  Only tests, the smoke check and
the bench's CPU baseline import it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libmoons_oracle.so")

from moons_b200.capi import BCSpec, ISP, SolveInfo, MHDParams, StepInfo  # noqa: E402  (plain ctypes structs)

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_lib = None


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("moons_oracle.cpp", "moons_oracle.hpp", "oracle_capi.cpp", "moons_oracle_mhd.cpp", "unet_oracle.cpp", "Makefile")]
    stale = not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs)
    if force or stale:
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        sig = {
            "or_last_error": (C.c_char_p, []),
            "or_mesh_create": (_P, [_D, C.c_int, _D, C.c_int, _D, C.c_int]),
            "or_mesh_destroy": (None, [_P]),
            "or_sf_create": (_P, [_P, C.c_int]),
            "or_sf_destroy": (None, [_P]),
            "or_sf_shape": (C.c_int, [_P, C.POINTER(C.c_int)]),
            "or_sf_upload": (C.c_int, [_P, _D, C.c_longlong]),
            "or_sf_download": (C.c_int, [_P, _D, C.c_longlong]),
            "or_sf_set_bcs": (C.c_int, [_P, C.POINTER(BCSpec)]),
            "or_apply_bcs": (C.c_int, [_P]),
            "or_apply_bcs_implicit": (C.c_int, [_P]),
            "or_del": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int]),
            "or_grad": (C.c_int, [_P, _P, _P, _P]),
            "or_div": (C.c_int, [_P, _P, _P, _P]),
            "or_curl": (C.c_int, [_P, _P, _P, _P, _P, _P]),
            "or_lap_centered": (C.c_int, [_P, _P]),
            "or_lap_uniform_coeff": (C.c_int, [_P, _P]),
            "or_lap_var": (C.c_int, [_P, _P, _P, _P, _P]),
            "or_interp": (C.c_int, [_P, _P, C.c_int]),
            "or_pcg_create": (_P, [C.c_int, C.c_int, C.c_int, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P),
                                   C.c_double]),
            "or_pcg_destroy": (None, [_P]),
            "or_pcg_update_mfp": (C.c_int, [_P, C.c_double, C.c_int]),
            "or_pcg_solve": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(ISP), C.POINTER(SolveInfo)]),
            "or_pcg_apply_op": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P)]),
            "or_clean_div": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), _P, C.c_double, C.POINTER(_P), _P,
                                       C.POINTER(ISP), C.POINTER(SolveInfo)]),
            "or_mhd_create": (_P, [_P, _P, C.POINTER(MHDParams)]),
            "or_mhd_destroy": (None, [_P]),
            "or_mhd_upload": (C.c_int, [_P, C.c_int, C.c_int, _D, C.c_longlong]),
            "or_mhd_download": (C.c_int, [_P, C.c_int, C.c_int, _D, C.c_longlong]),
            "or_mhd_shape": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_int)]),
            "or_mhd_init": (C.c_int, [_P]),
            "or_mhd_step": (C.c_int, [_P, C.c_int, C.POINTER(StepInfo)]),
            "or_mhd_divergence": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
            "or_unet_layer": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                        _F, _F, _F, _F, C.c_int, _F]),
            "or_unet_nparams": (C.c_longlong, []),
            "or_unet_set_exact": (None, [C.c_int]),
            "or_unet_adam": (None, [_F, _F, _F, _F, C.c_longlong, C.c_float, C.c_int]),
            "or_unet_forward": (C.c_int, [C.c_int, C.c_int, C.c_int, _F, C.c_double, _D, _F, _D]),
            "or_unet_loss_grad": (C.c_int, [C.c_int, C.c_int, C.c_int, _F, C.c_double, _D, _F, _D, C.c_int, _D, _D,
                                            _D, C.c_double, _D, _F]),
        }
        for n, (rt, at) in sig.items():
            f = getattr(L, n)
            f.restype = rt
            f.argtypes = at
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def threads() -> int:
    """Host threads the oracle's loops run on (MOONS_ORACLE_THREADS, default all)."""
    f = lib().or_threads
    f.restype = C.c_int
    return int(f())


def _check(code):
    if code != 0:
        raise OracleError(f"oracle error {code}: {lib().or_last_error().decode()}")


class Mesh:
    def __init__(self, hx, hy, hz, device: int = -1):
        self._keep = [np.ascontiguousarray(h, dtype=np.float64) for h in (hx, hy, hz)]
        k = self._keep
        self.h = lib().or_mesh_create(k[0].ctypes.data_as(_D), len(k[0]), k[1].ctypes.data_as(_D), len(k[1]),
                                      k[2].ctypes.data_as(_D), len(k[2]))
        if not self.h:
            raise OracleError(lib().or_last_error().decode())
        self.sn = tuple(len(x) for x in k)

    def field(self, dl):
        return Field(self, dl)

    def sync(self):
        pass

    def __del__(self):
        try:
            if self.h:
                lib().or_mesh_destroy(self.h)
                self.h = None
        except Exception:
            pass


class Field:
    def __init__(self, mesh: Mesh, dl: int):
        self.mesh = mesh
        self.dl = dl
        self.h = lib().or_sf_create(mesh.h, dl)
        s = (C.c_int * 3)()
        lib().or_sf_shape(self.h, s)
        self.shape = (s[0], s[1], s[2])

    @property
    def n(self):
        return self.shape[0] * self.shape[1] * self.shape[2]

    def upload(self, a):
        a = np.asarray(a, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        flat = np.ascontiguousarray(a.ravel(order="F"))
        _check(lib().or_sf_upload(self.h, flat.ctypes.data_as(_D), flat.size))

    def download(self):
        flat = np.empty(self.n)
        _check(lib().or_sf_download(self.h, flat.ctypes.data_as(_D), flat.size))
        return flat.reshape(self.shape, order="F")

    def fill(self, v):
        self.upload(np.full(self.shape, float(v)))

    def set_bcs(self, spec):
        _check(lib().or_sf_set_bcs(self.h, C.byref(spec)))

    def apply_bcs(self):
        _check(lib().or_apply_bcs(self.h))

    def apply_bcs_implicit(self):
        _check(lib().or_apply_bcs_implicit(self.h))

    def __del__(self):
        try:
            if self.h:
                lib().or_sf_destroy(self.h)
                self.h = None
        except Exception:
            pass


def delta(out, inp, n, d, pad, gen):
    _check(lib().or_del(out.h, inp.h, n, d, pad, gen))


def grad(gx, gy, gz, u):
    _check(lib().or_grad(gx.h, gy.h, gz.h, u.h))


def div(o, ux, uy, uz):
    _check(lib().or_div(o.h, ux.h, uy.h, uz.h))


def curl(o, u):
    _check(lib().or_curl(o[0].h, o[1].h, o[2].h, u[0].h, u[1].h, u[2].h))


def lap_centered(o, u):
    _check(lib().or_lap_centered(o.h, u.h))


def lap_uniform_coeff(o, u):
    _check(lib().or_lap_uniform_coeff(o.h, u.h))


def lap_var(o, u, k):
    _check(lib().or_lap_var(o.h, u.h, k[0].h, k[1].h, k[2].h))


def interp(o, i, d):
    _check(lib().or_interp(o.h, i.h, d))


def _ptrs(fs):
    arr = (_P * 3)()
    for i, f in enumerate(fs):
        arr[i] = f.h if f is not None else None
    return arr


class PCG:
    def __init__(self, mesh, op, prec, x: Sequence[Field], x_bc: Sequence[Field], k=None, coeff_implicit=0.0):
        self.mesh = mesh
        self.nc = len(x)
        self.h = lib().or_pcg_create(op, prec, self.nc, _ptrs(x), _ptrs(x_bc), _ptrs(k) if k is not None else None,
                                     float(coeff_implicit))
        if not self.h:
            raise OracleError(lib().or_last_error().decode())

    def update_mfp(self, coeff, update_prec=True):
        _check(lib().or_pcg_update_mfp(self.h, float(coeff), 1 if update_prec else 0))

    def apply_op(self, out, x):
        """out = A x with the solver's operator_explicit (matrix_free_operators.f90)."""
        _check(lib().or_pcg_apply_op(self.h, _ptrs(out), _ptrs(x)))

    def solve(self, x, b, params):
        info = SolveInfo()
        _check(lib().or_pcg_solve(self.h, _ptrs(x), _ptrs(b), C.byref(params), C.byref(info)))
        return info.as_dict()

    def __del__(self):
        try:
            if self.h:
                lib().or_pcg_destroy(self.h)
                self.h = None
        except Exception:
            pass


def clean_div(pcg, X, Xstar, phi, scale, temp_F, temp_CC, params) -> dict:
    """clean_div (clean_divergence.f90:37-59) with the solver pcg."""
    info = SolveInfo()
    _check(lib().or_clean_div(pcg.h, _ptrs(X), _ptrs(Xstar), phi.h, float(scale), _ptrs(temp_F), temp_CC.h,
                              C.byref(params), C.byref(info)))
    return info.as_dict()


class MHD:
    """The oracle's MHD time step, same surface as moons_b200.capi.MHD."""

    def __init__(self, mesh_mom, mesh_ind, params):
        self.meshes = (mesh_mom, mesh_ind)
        self.params = params
        self.h = lib().or_mhd_create(mesh_mom.h, mesh_ind.h, C.byref(params))
        if not self.h:
            raise ValueError("or_mhd_create: solve_method_U and solve_method_B must be 0 to 9, rk_stages 0, 1 "
                             "or 3, solve_method_T 1 to 5")

    def shape(self, which, comp=0):
        s = (C.c_int * 3)()
        _check(lib().or_mhd_shape(self.h, which, comp, s))
        return (s[0], s[1], s[2])

    def upload(self, which, comp, a):
        a = np.asarray(a, dtype=np.float64)
        assert a.shape == self.shape(which, comp)
        flat = np.ascontiguousarray(a.ravel(order="F"))
        _check(lib().or_mhd_upload(self.h, which, comp, flat.ctypes.data_as(_D), flat.size))

    def download(self, which, comp=0):
        shp = self.shape(which, comp)
        flat = np.empty(shp[0] * shp[1] * shp[2])
        _check(lib().or_mhd_download(self.h, which, comp, flat.ctypes.data_as(_D), flat.size))
        return flat.reshape(shp, order="F")

    def init(self):
        _check(lib().or_mhd_init(self.h))

    def step(self, n=1):
        info = StepInfo()
        _check(lib().or_mhd_step(self.h, int(n), C.byref(info)))
        return info.as_dict()

    def divergence(self):
        a, b = C.c_double(), C.c_double()
        _check(lib().or_mhd_divergence(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def __del__(self):
        try:
            if self.h:
                lib().or_mhd_destroy(self.h)
                self.h = None
        except Exception:
            pass


# ---- learned preconditioner (U-Net) restatement ------------------------------
def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _fptr(a):
    return None if a is None else a.ctypes.data_as(_F)


def unet_layer(op, X, Y, Z, cinA, cinB, cout, inp=None, dout=None, W=None, bias=None, relu=True):
    """One U-Net layer on the CPU (same contract as capi.unet_layer_check)."""
    cin = cinA + cinB
    inp, dout, W, bias = _f32(inp), _f32(dout), _f32(W), _f32(bias)
    n = {0: cout * X * Y * Z, 1: cin * X * Y * Z, 2: cout * cin * 27 + cout}[op]
    out = np.empty(n, dtype=np.float32)
    _check(lib().or_unet_layer(op, X, Y, Z, cinA, cinB, cout, _fptr(inp), _fptr(dout), _fptr(W), _fptr(bias),
                               int(relu), _fptr(out)))
    return out


def unet_set_exact(on: bool):
    """Exact arithmetic (no BF16 rounding) in the U-Net restatement."""
    lib().or_unet_set_exact(int(bool(on)))


def unet_adam(w, g, m, v, lr: float, t: int):
    """One Adam step on FP32 arrays (w, m, v updated in place), the CPU
    statement of the library's training-step update."""
    for a in (w, g, m, v):
        assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    lib().or_unet_adam(_fptr(w), _fptr(g), _fptr(m), _fptr(v), C.c_longlong(w.size), C.c_float(lr), int(t))


def unet_nparams() -> int:
    return int(lib().or_unet_nparams())


def _cc(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))


def unet_forward(X, Y, Z, params, out_scale, r, feat=None):
    """z = M(r) of the network with the given flat parameters; r, feat and
    the result are cell-centred arrays with ghosts (Fortran order)."""
    p = _f32(params)
    rr = _cc(r)
    ff = None if feat is None else np.ascontiguousarray(np.asarray(feat, dtype=np.float32).ravel(order="F"))
    z = np.zeros_like(rr)
    _check(lib().or_unet_forward(X, Y, Z, _fptr(p), float(out_scale), rr.ctypes.data_as(_D), _fptr(ff),
                                 z.ctypes.data_as(_D)))
    return z.reshape((X + 2, Y + 2, Z + 2), order="F")


def unet_loss_grad(X, Y, Z, params, out_scale, r, e, feat=None, kind=1, k=None, h=1.0):
    """Loss (kind 0 relative L2, 1 cosine, 2 energy-norm cosine with the
    uniform-mesh all-Neumann operator of face coefficients k and spacing h)
    and its gradient."""
    p = _f32(params)
    rr, ee = _cc(r), _cc(e)
    ff = None if feat is None else np.ascontiguousarray(np.asarray(feat, dtype=np.float32).ravel(order="F"))
    loss = np.zeros(1, dtype=np.float64)
    g = np.zeros(p.size, dtype=np.float32)
    kf = [None] * 3 if k is None else [_cc(a) for a in k]
    kk = [None if a is None else a.ctypes.data_as(_D) for a in kf]
    _check(lib().or_unet_loss_grad(X, Y, Z, _fptr(p), float(out_scale), rr.ctypes.data_as(_D), _fptr(ff),
                                   ee.ctypes.data_as(_D), int(kind), *kk, float(h), loss.ctypes.data_as(_D),
                                   _fptr(g)))
    return float(loss[0]), g
