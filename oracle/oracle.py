"""ctypes front end of the CPU oracle (oracle/kirchhoff_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

Functions take and return numpy arrays in the reference's SoA argument order
(crates/xrt-python/src/lib.rs:321-393, ``diffraction_integral_rs``):
rays = (x, y, z, nx, ny, nz, nl, es_re, es_im, ep_re, ep_im, energy),
pixels = (x, y, z); result = (es_re, es_im, ep_re, ep_im).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

RAY_FIELDS = ("x", "y", "z", "nx", "ny", "nz", "nl", "es_re", "es_im", "ep_re", "ep_im", "energy")
PIX_FIELDS = ("x", "y", "z")


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        d = ctypes.POINTER(ctypes.c_double)
        f = ctypes.POINTER(ctypes.c_float)
        sz = ctypes.c_size_t
        for name in ("oracle_kahan_f64", "oracle_plain_f64", "oracle_kahan_ld"):
            fn = getattr(lib, name)
            fn.argtypes = [d] * 12 + [sz] + [d] * 3 + [sz] + [d] * 4 + [ctypes.c_int]
            fn.restype = None
        lib.oracle_wgsl_f32.argtypes = [f] * 12 + [sz] + [f] * 3 + [sz] + [d] * 4 + [ctypes.c_int]
        lib.oracle_wgsl_f32.restype = None
        lib.oracle_max_threads.restype = ctypes.c_int
        lib.oracle_prepare_wave.argtypes = [d, ctypes.c_double, ctypes.c_double, sz, sz, d, d, d]
        lib.oracle_prepare_wave.restype = None
        pp = ctypes.POINTER(d)
        lib.oracle_beam_rays.argtypes = [pp, d, ctypes.POINTER(sz), sz, pp]
        lib.oracle_beam_rays.restype = None
        lib.oracle_fresnel.argtypes = ([d] * 4 + [sz] + [ctypes.c_double] * 4 + [sz]
                                       + [ctypes.c_double] * 2 + [sz, d, d, ctypes.c_int])
        lib.oracle_fresnel.restype = None
        _lib = lib
    return _lib


def max_threads() -> int:
    return int(_load().oracle_max_threads())


def _as(arr, dtype):
    a = np.ascontiguousarray(np.asarray(arr, dtype=dtype))
    return a


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _run(fn_name, rays, pixels, dtype, threads):
    lib = _load()
    ctype = ctypes.c_double if dtype == np.float64 else ctypes.c_float
    r = [_as(a, dtype) for a in rays]
    p = [_as(a, dtype) for a in pixels]
    n = len(r[0])
    m = len(p[0])
    if any(len(a) != n for a in r) or any(len(a) != m for a in p):
        raise ValueError("array length mismatch")
    out = [np.zeros(m, dtype=np.float64) for _ in range(4)]
    getattr(lib, fn_name)(*[_ptr(a, ctype) for a in r], n, *[_ptr(a, ctype) for a in p], m,
                          *[_ptr(a, ctypes.c_double) for a in out], int(threads))
    return tuple(out)


def kahan_f64(rays, pixels, threads: int = 0):
    """src/waves/diffraction.rs:56-117 restated (the correctness oracle)."""
    return _run("oracle_kahan_f64", rays, pixels, np.float64, threads)


def kahan_ld(rays, pixels, threads: int = 0):
    """kahan_f64 with the phase k*|p - r| in x87 extended precision: the
    formula's value without FP64's phase rounding (which reaches 1e-4 rad at
    k*path ~ 1e12)."""
    return _run("oracle_kahan_ld", rays, pixels, np.float64, threads)


def plain_f64(rays, pixels, threads: int = 0):
    """src/gpu/fallback.rs:29-71 restated (plain f64 sum, no Kahan)."""
    return _run("oracle_plain_f64", rays, pixels, np.float64, threads)


def wgsl_f32(gpu_rays, pixels, threads: int = 0):
    """src/gpu/shaders/kirchhoff.wgsl:56-135 + src/gpu/kirchhoff.rs:96-297.

    ``gpu_rays`` follows the GpuRay field order (kirchhoff.rs:20-35):
    (x, y, z, nx, ny, nz, nl, energy, es_re, es_im, ep_re, ep_im).
    """
    return _run("oracle_wgsl_f32", gpu_rays, pixels, np.float32, threads)


def prepare_wave(center, dx, dz, nx, nz):
    """src/waves/prepare_wave.rs:40-68 restated: (x, y, z) of nx*nz points,
    x outer, z inner."""
    lib = _load()
    c = _as(center, np.float64)
    m = int(nx) * int(nz)
    out = [np.empty(m, dtype=np.float64) for _ in range(3)]
    lib.oracle_prepare_wave(_ptr(c, ctypes.c_double), float(dx), float(dz), int(nx), int(nz),
                            *[_ptr(a, ctypes.c_double) for a in out])
    return tuple(out)


BEAM_FIELDS = ("x", "y", "z", "a", "b", "c", "e", "es_re", "es_im", "ep_re", "ep_im")


def beam_to_rays(beam, normals, good):
    """src/waves/prepare_wave.rs:78-111 restated. ``beam`` maps BEAM_FIELDS to
    arrays (amplitude keys absent: es = 1, ep = 0); ``normals`` is (n, 3);
    returns the 12 ray columns."""
    lib = _load()
    cols = [_as(beam[k], np.float64) if k in beam else None for k in BEAM_FIELDS]
    nrm = _as(normals, np.float64).reshape(-1)
    g = np.ascontiguousarray(np.asarray(good, dtype=np.uint64))
    if len(g) and int(g.max()) >= len(cols[0]):
        raise IndexError("good index out of range")
    out = [np.empty(len(g), dtype=np.float64) for _ in range(12)]
    dp = ctypes.POINTER(ctypes.c_double)
    beam_arr = (dp * 11)(*[(_ptr(a, ctypes.c_double) if a is not None else dp()) for a in cols])
    out_arr = (dp * 12)(*[_ptr(a, ctypes.c_double) for a in out])
    lib.oracle_beam_rays(beam_arr, _ptr(nrm, ctypes.c_double),
                         g.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t)), len(g), out_arr)
    return tuple(out)


def fresnel(ray_x, ray_z, es_re, es_im, energy, dist, x_min, x_max, nx, z_min, z_max, nz,
            threads: int = 0):
    """src/waves/fresnel.rs:53-106 restated: (re, im) of nx*nz amplitudes,
    index iz * nx + ix."""
    lib = _load()
    cols = [_as(a, np.float64) for a in (ray_x, ray_z, es_re, es_im)]
    n = len(cols[0])
    if any(len(a) != n for a in cols):
        raise ValueError("array length mismatch")
    m = int(nx) * int(nz)
    out = [np.zeros(m, dtype=np.float64) for _ in range(2)]
    lib.oracle_fresnel(*[_ptr(a, ctypes.c_double) for a in cols], n, float(energy), float(dist),
                       float(x_min), float(x_max), int(nx), float(z_min), float(z_max), int(nz),
                       *[_ptr(a, ctypes.c_double) for a in out], int(threads))
    return tuple(out)
