"""Screens and rays from a beam: the producers in front of the Kirchhoff path.

Mirrors ``waves::prepare_wave`` (src/waves/prepare_wave.rs): ``WaveParams``
(:11-23), ``prepare_wave`` (:40-68, x outer, z inner) and
``beam_to_diffraction_rays`` (:78-111, nl = n . (a, b, c), es = 1 and ep = 0
for a beam without amplitudes). All three run on the device in libxk.so;
``diffraction_from_beam`` chains them with the integral so the beam's
columns are uploaded once and neither the rays nor the screen make a host
round trip.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import _path, _require_ctx, _f64, _ptr, RAY_FIELDS

BEAM_FIELDS = ("x", "y", "z", "a", "b", "c", "e")
AMPLITUDE_FIELDS = ("es_re", "es_im", "ep_re", "ep_im")


@dataclass
class WaveParams:
    """Screen centre [mm], half-widths dx, dz [mm], points nx, nz."""
    center: tuple
    dx: float
    dz: float
    nx: int
    nz: int

    def _c(self):
        if self.nx < 0 or self.nz < 0:
            raise ValueError("nx and nz must be non-negative")
        c = (ctypes.c_double * 3)(*[float(v) for v in self.center])
        return _lib.XkWaveParams(c, float(self.dx), float(self.dz), int(self.nx), int(self.nz))


def prepare_wave(params: WaveParams, ctx=None):
    """(x, y, z) of the nx*nz screen points, index ix*nz + iz."""
    m = int(params.nx) * int(params.nz)
    out = [np.empty(m, dtype=np.float64) for _ in range(3)]
    if m == 0:
        return tuple(out)
    ctx = _require_ctx(ctx)
    xo = _lib.XkPixelsOut(*[_ptr(a) for a in out])
    wp = params._c()
    _lib.check(_lib.load().xk_prepare_wave(ctx.handle, ctypes.byref(wp), ctypes.byref(xo)),
               ctx.handle)
    return tuple(out)


def _beam_args(beam, normals, good):
    cols = [_f64(beam[k]) for k in BEAM_FIELDS]
    n = len(cols[0])
    for k, a in zip(BEAM_FIELDS, cols):
        if len(a) != n:
            raise ValueError(f"array length mismatch: beam {k} has {len(a)} elements, x has {n}")
    have = [k in beam and beam[k] is not None for k in AMPLITUDE_FIELDS]
    if any(have) and not all(have):
        raise ValueError("amplitudes must be given all four or none")
    amps = [_f64(beam[k]) for k in AMPLITUDE_FIELDS] if all(have) else []
    if any(len(a) != n for a in amps):
        raise ValueError("array length mismatch in the beam amplitudes")
    nrm = _f64(normals).reshape(-1)
    if len(nrm) != 3 * n:
        raise ValueError("normals must hold 3 values per beam ray")
    g = np.ascontiguousarray(np.asarray(good, dtype=np.uint64)).astype(np.uintp, copy=False)
    keep = cols + amps + [nrm, g]
    ptrs = [_ptr(a) for a in cols] + ([_ptr(a) for a in amps] if amps else [_lib._dp()] * 4)
    xb = _lib.XkBeam(*ptrs)
    return xb, n, nrm, g, keep


def beam_to_diffraction_rays(beam, normals, good, ctx=None):
    """Rays (dict of RAY_FIELDS arrays) of the beam rays listed in ``good``.

    ``beam``: mapping with x, y, z, a, b, c, e and optionally es_re, es_im,
    ep_re, ep_im; ``normals``: (n, 3) surface normals of every beam ray.
    An index out of range raises XkError (the reference panics)."""
    xb, n, nrm, g, keep = _beam_args(beam, normals, good)
    out = [np.empty(len(g), dtype=np.float64) for _ in range(12)]
    if len(g) == 0:
        return dict(zip(RAY_FIELDS, out))
    ctx = _require_ctx(ctx)
    xo = _lib.XkRaysOut(*[_ptr(a) for a in out])
    gp = g.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t))
    rc = _lib.load().xk_beam_to_rays(ctx.handle, ctypes.byref(xb), n, _ptr(nrm), gp, len(g),
                                     ctypes.byref(xo))
    _lib.check(rc, ctx.handle)
    del keep
    return dict(zip(RAY_FIELDS, out))


def diffraction_from_beam(beam, normals, good, params: WaveParams, path="f32pr", ctx=None,
                          return_stats=False):
    """beam -> rays -> screen -> Kirchhoff integral, all on the device.
    Returns (es_re, es_im, ep_re, ep_im) over the screen of ``params``."""
    path_code = _path(path)
    xb, n, nrm, g, keep = _beam_args(beam, normals, good)
    m = int(params.nx) * int(params.nz)
    out = [np.zeros(m, dtype=np.float64) for _ in range(4)]
    ctx = _require_ctx(ctx)
    xf = _lib.XkField(*[_ptr(a) for a in out])
    wp = params._c()
    st = _lib.XkStats()
    gp = g.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t))
    rc = _lib.load().xk_diffraction_beam(ctx.handle, ctypes.byref(xb), n, _ptr(nrm), gp, len(g),
                                         ctypes.byref(wp), ctypes.byref(xf), path_code,
                                         ctypes.byref(st))
    _lib.check(rc, ctx.handle)
    del keep
    if return_stats:
        return tuple(out), st.to_dict()
    return tuple(out)
