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
