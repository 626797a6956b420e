"""2-D Fresnel propagation: mirror of ``waves::fresnel`` (src/waves/fresnel.rs).

``FresnelScreen`` (:14-27), ``FresnelResult`` (:30-48, with ``intensity()``)
and ``fresnel_propagate`` (:53-106) keep the reference's names, fields and
output order (index iz * nx + ix). The sum runs in libxk.so:

* ``path="separable"`` (default): the Fresnel kernel factorises over the
  regular screen, so the whole screen is one complex matrix product over the
  rays, computed on the tensor cores from FP64 phasors split into f16
  hi + lo parts (relative L2 error ~5e-6 against the FP64 sum);
* ``path="f64"``: the reference's FP64 sum, term for term.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import _require_ctx, _f64, _ptr

_FRESNEL_PATHS = {"separable": _lib.XK_PATH_SEPARABLE, "f64": _lib.XK_PATH_F64,
                  _lib.XK_PATH_SEPARABLE: _lib.XK_PATH_SEPARABLE, _lib.XK_PATH_F64: _lib.XK_PATH_F64}


@dataclass
class FresnelScreen:
    x_min: float
    x_max: float
    nx: int
    z_min: float
    z_max: float
    nz: int


@dataclass
class FresnelResult:
    amplitude: np.ndarray  # complex128, nx * nz, index iz * nx + ix
    x_pixels: np.ndarray
    z_pixels: np.ndarray
    nx: int
    nz: int

    def intensity(self) -> np.ndarray:
        return np.abs(self.amplitude) ** 2


def fresnel_propagate(ray_x, ray_z, ray_es, energy: float, dist: float, screen: FresnelScreen,
                      path="separable", ctx=None, return_stats=False):
    """Propagate rays at (x, z) with complex amplitudes ``ray_es`` (a complex
    array, or a (re, im) pair of float64 arrays) to the screen at distance
    ``dist`` [mm]; ``energy`` in eV."""
    if path not in _FRESNEL_PATHS:
        raise ValueError(f"unknown path {path!r} (separable or f64)")
    code = _FRESNEL_PATHS[path]
    x, z = _f64(ray_x), _f64(ray_z)
    if isinstance(ray_es, tuple) and len(ray_es) == 2:
        er, ei = _f64(ray_es[0]), _f64(ray_es[1])  # (re, im) arrays, used in place
    else:
        es = np.asarray(ray_es, dtype=np.complex128)
        er, ei = np.ascontiguousarray(es.real), np.ascontiguousarray(es.imag)
    if not (len(x) == len(z) == len(er) == len(ei)):
        raise ValueError("array length mismatch: ray_x, ray_z and ray_es differ in length")
    if screen.nx < 0 or screen.nz < 0:
        raise ValueError("nx and nz must be non-negative")
    nx, nz = int(screen.nx), int(screen.nz)
    m = nx * nz
    re = np.zeros(m, dtype=np.float64)
    im = np.zeros(m, dtype=np.float64)
    xp = np.zeros(nx, dtype=np.float64)
    zp = np.zeros(nz, dtype=np.float64)
    st = _lib.XkStats()
    if m:
        ctx = _require_ctx(ctx)
        sc = _lib.XkFresnelScreen(float(screen.x_min), float(screen.x_max), nx,
                                  float(screen.z_min), float(screen.z_max), nz)
        rc = _lib.load().xk_fresnel_propagate(
            ctx.handle, _ptr(x), _ptr(z), _ptr(er), _ptr(ei), len(x), float(energy), float(dist),
            ctypes.byref(sc), _ptr(re), _ptr(im), _ptr(xp), _ptr(zp), code, ctypes.byref(st))
        _lib.check(rc, ctx.handle)
    res = FresnelResult(re + 1j * im, xp, zp, nx, nz)
    if return_stats:
        return res, st.to_dict()
    return res
