"""Kirchhoff diffraction on B200, behind the xrt-rs interface.

Drop-in for the Kirchhoff path of physwkim/xrt-rs:

* ``diffraction_integral_rs(15 lists) -> 4 lists`` mirrors the PyO3 binding
  (crates/xrt-python/src/lib.rs:321-393), including its ValueError on
  mismatched array lengths (lib.rs:31-45).
* ``diffraction_integral(rays, pixels)`` is the numpy form of
  waves::diffraction::diffraction_integral (src/waves/diffraction.rs:56-64).
* ``GpuContext``, ``kirchhoff_gpu`` and ``kirchhoff_auto`` mirror
  src/gpu/context.rs, src/gpu/kirchhoff.rs:77-83 and src/gpu/fallback.rs:19-26,
  with GpuRay / GpuPixel as numpy structured dtypes of the same layout.

All compute runs in libxk.so (CUDA, sm_100a). There is no CPU fallback: with
no CUDA device every compute call raises XkError (code XK_ERR_NO_DEVICE).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import XkError, XK_PATH_F64, XK_PATH_F32PR  # noqa: F401

__all__ = [
    "diffraction_integral_rs", "diffraction_integral", "diffraction_integral_device",
    "GpuContext", "kirchhoff_gpu", "kirchhoff_auto", "GPU_RAY_DTYPE", "GPU_PIXEL_DTYPE",
    "XkError", "XK_PATH_F64", "XK_PATH_F32PR", "RAY_FIELDS", "PIXEL_FIELDS", "Batch",
    "autotune", "WaveParams", "prepare_wave", "beam_to_diffraction_rays", "diffraction_from_beam",
    "FresnelScreen", "FresnelResult", "fresnel_propagate", "route_reason",
]

RAY_FIELDS = ("x", "y", "z", "nx", "ny", "nz", "nl", "es_re", "es_im", "ep_re", "ep_im", "energy")
PIXEL_FIELDS = ("x", "y", "z")
FIELD_FIELDS = ("es_re", "es_im", "ep_re", "ep_im")

# GpuRay (src/gpu/kirchhoff.rs:20-35) and GpuPixel (:38-45).
GPU_RAY_DTYPE = np.dtype([(n, np.float32) for n in
                          ("x", "y", "z", "nx", "ny", "nz", "nl", "energy",
                           "es_re", "es_im", "ep_re", "ep_im")])
GPU_PIXEL_DTYPE = np.dtype([(n, np.float32) for n in ("x", "y", "z", "_pad")])

_PATHS = {"f64": XK_PATH_F64, "f32pr": XK_PATH_F32PR, XK_PATH_F64: XK_PATH_F64,
          XK_PATH_F32PR: XK_PATH_F32PR}


def route_reason(code: int) -> str:
    """Why an f32pr request ran on the FP64 path (stats ``routed_reason``)."""
    return _lib.load().xk_route_reason(int(code)).decode()


def _path(path) -> int:
    try:
        return _PATHS[path]
    except KeyError:
        raise ValueError(f"unknown path {path!r}; use 'f64' or 'f32pr'") from None


class GpuContext:
    """A CUDA device context (gpu::context::GpuContext)."""

    def __init__(self, handle, owned: bool):
        self._h = handle
        self._owned = owned

    @classmethod
    def new(cls, device: int = 0):
        """GpuContext::new: None when no CUDA device exists."""
        lib = _lib.load()
        h = ctypes.c_void_p()
        rc = lib.xk_init(device, ctypes.byref(h))
        if rc == _lib.XK_ERR_NO_DEVICE:
            return None
        _lib.check(rc)
        return cls(h, True)

    @classmethod
    def shared(cls):
        """GpuContext::shared: the process-wide context, or None."""
        lib = _lib.load()
        h = ctypes.c_void_p()
        rc = lib.xk_shared(ctypes.byref(h))
        if rc == _lib.XK_ERR_NO_DEVICE or not h.value:
            return None
        _lib.check(rc)
        return cls(h, False)

    def set_option(self, name: str, value: float):
        """Tuning knob of the F32PR path (phase_budget, sweep, groups, items_per_warp)."""
        _lib.check(_lib.load().xk_set_option(self._h, name.encode(), float(value)), self._h)

    def adapter_name(self) -> str:
        return _lib.load().xk_device_name(self._h).decode()

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._owned and self._h:
            _lib.load().xk_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _require_ctx(ctx):
    if ctx is None:
        ctx = GpuContext.shared()
        if ctx is None:
            raise XkError(_lib.XK_ERR_NO_DEVICE, "no CUDA device")
    return ctx


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check_lengths(pairs):
    # Same message shape as check_equal_lengths (crates/xrt-python/src/lib.rs:31-45).
    if len(pairs) < 2:
        return
    ref_name, ref_len = pairs[0]
    for name, n in pairs[1:]:
        if n != ref_len:
            raise ValueError(f"array length mismatch: {name} has {n} elements but "
                             f"{ref_name} has {ref_len}")


def diffraction_integral(rays, pixels, path="f64", ctx=None, return_stats=False):
    """Kirchhoff integral for numpy inputs.

    ``rays``: mapping or sequence of the 12 per-ray arrays in RAY_FIELDS order;
    ``pixels``: mapping or sequence of (x, y, z). Returns four float64 arrays
    (es_re, es_im, ep_re, ep_im), plus a stats dict when ``return_stats``.
    """
    path_code = _path(path)
    if isinstance(rays, dict):
        rays = [rays[k] for k in RAY_FIELDS]
    if isinstance(pixels, dict):
        pixels = [pixels[k] for k in PIXEL_FIELDS]
    r = [_f64(a) for a in rays]
    p = [_f64(a) for a in pixels]
    if len(r) != 12 or len(p) != 3:
        raise ValueError("expected 12 ray arrays and 3 pixel arrays")
    _check_lengths([("ray_" + n, len(a)) for n, a in zip(RAY_FIELDS, r)])
    _check_lengths([("pix_" + n, len(a)) for n, a in zip(PIXEL_FIELDS, p)])
    n, m = len(r[0]), len(p[0])
    out = [np.zeros(m, dtype=np.float64) for _ in range(4)]
    ctx = _require_ctx(ctx)
    lib = _lib.load()
    xr = _lib.XkRays(*[_ptr(a) for a in r])
    xp = _lib.XkPixels(*[_ptr(a) for a in p])
    xf = _lib.XkField(*[_ptr(a) for a in out])
    st = _lib.XkStats()
    rc = lib.xk_diffraction_integral(ctx.handle, ctypes.byref(xr), n, ctypes.byref(xp), m,
                                     ctypes.byref(xf), path_code, ctypes.byref(st))
    _lib.check(rc, ctx.handle)
    if return_stats:
        return tuple(out), st.to_dict()
    return tuple(out)


def diffraction_integral_rs(ray_x, ray_y, ray_z, ray_nx, ray_ny, ray_nz, ray_nl,
                            ray_es_re, ray_es_im, ray_ep_re, ray_ep_im, ray_energy,
                            pix_x, pix_y, pix_z, path="f64"):
    """Mirror of xrt_rs.diffraction_integral_rs (crates/xrt-python/src/lib.rs:321-393).

    15 sequences in, (es_re, es_im, ep_re, ep_im) lists out. Raises
    ValueError on mismatched lengths, like the reference binding.
    """
    rays = [ray_x, ray_y, ray_z, ray_nx, ray_ny, ray_nz, ray_nl, ray_es_re, ray_es_im,
            ray_ep_re, ray_ep_im, ray_energy]
    _check_lengths([("ray_" + n, len(a)) for n, a in zip(RAY_FIELDS, rays)])
    _check_lengths([("pix_x", len(pix_x)), ("pix_y", len(pix_y)), ("pix_z", len(pix_z))])
    out = diffraction_integral(rays, [pix_x, pix_y, pix_z], path=path)
    return tuple(o.tolist() for o in out)


def diffraction_integral_device(rays, pixels, out, path="f32pr", ctx=None, stream=None):
    """Device-resident form: every array is an object with ``data_ptr()``
    (e.g. a contiguous float64 CUDA tensor). Returns the stats dict."""
    ctx = _require_ctx(ctx)
    lib = _lib.load()
    dp = ctypes.POINTER(ctypes.c_double)

    def cast(t):
        return ctypes.cast(ctypes.c_void_p(int(t.data_ptr())), dp)

    if isinstance(rays, dict):
        rays = [rays[k] for k in RAY_FIELDS]
    if isinstance(pixels, dict):
        pixels = [pixels[k] for k in PIXEL_FIELDS]
    if isinstance(out, dict):
        out = [out[k] for k in FIELD_FIELDS]
    n = int(rays[0].numel()) if hasattr(rays[0], "numel") else len(rays[0])
    m = int(pixels[0].numel()) if hasattr(pixels[0], "numel") else len(pixels[0])
    xr = _lib.XkRays(*[cast(a) for a in rays])
    xp = _lib.XkPixels(*[cast(a) for a in pixels])
    xf = _lib.XkField(*[cast(a) for a in out])
    st = _lib.XkStats()
    s = ctypes.c_void_p(int(stream)) if stream is not None else None
    rc = lib.xk_diffraction_integral_device(ctx.handle, ctypes.byref(xr), n, ctypes.byref(xp), m,
                                            ctypes.byref(xf), _path(path), s, ctypes.byref(st))
    _lib.check(rc, ctx.handle)
    return st.to_dict()


class Batch:
    """Many independent solves in one persistent launch (xk_batch_*).

    ``solves`` is a sequence of (rays, pixels) pairs in the layout
    ``diffraction_integral`` takes. The inputs are copied to the device and
    planned once; ``run()`` replays the captured launch sequence and returns
    one (es_re, es_im, ep_re, ep_im) tuple per solve.
    """

    def __init__(self, solves, path="f32pr", ctx=None, graph=True, device_outputs=None):
        """With ``device_outputs`` (one 4-tuple of device tensors per solve),
        every array in ``solves`` must be a device tensor (``data_ptr()``) and
        results stay on the device."""
        self._ctx = _require_ctx(ctx)
        lib = _lib.load()
        self._keep = []
        self.outputs = []
        arr = (_lib.XkSolve * max(1, len(solves)))()
        if device_outputs is not None:
            dp = ctypes.POINTER(ctypes.c_double)

            def cast(t):
                return ctypes.cast(ctypes.c_void_p(int(t.data_ptr())), dp)

            for i, ((rays, pixels), outs) in enumerate(zip(solves, device_outputs)):
                if isinstance(rays, dict):
                    rays = [rays[k] for k in RAY_FIELDS]
                if isinstance(pixels, dict):
                    pixels = [pixels[k] for k in PIXEL_FIELDS]
                arr[i].rays = _lib.XkRays(*[cast(a) for a in rays])
                arr[i].n_rays = int(rays[0].numel())
                arr[i].pixels = _lib.XkPixels(*[cast(a) for a in pixels])
                arr[i].n_pix = int(pixels[0].numel())
                arr[i].out = _lib.XkField(*[cast(a) for a in outs])
                self.outputs.append(tuple(outs))
            flags = _lib.XK_BATCH_DEVICE | (0 if graph else _lib.XK_BATCH_NO_GRAPH)
            h = ctypes.c_void_p()
            rc = lib.xk_batch_create(self._ctx.handle, arr, len(solves), _path(path), flags,
                                     ctypes.byref(h))
            _lib.check(rc, self._ctx.handle)
            self._arr = arr
            self._h = h
            self.n = len(solves)
            return
        for i, (rays, pixels) in enumerate(solves):
            if isinstance(rays, dict):
                rays = [rays[k] for k in RAY_FIELDS]
            if isinstance(pixels, dict):
                pixels = [pixels[k] for k in PIXEL_FIELDS]
            r = [_f64(a) for a in rays]
            p = [_f64(a) for a in pixels]
            _check_lengths([("ray_" + n, len(a)) for n, a in zip(RAY_FIELDS, r)])
            _check_lengths([("pix_" + n, len(a)) for n, a in zip(PIXEL_FIELDS, p)])
            o = [np.zeros(len(p[0]), dtype=np.float64) for _ in range(4)]
            self._keep += r + p
            self.outputs.append(tuple(o))
            arr[i].rays = _lib.XkRays(*[_ptr(a) for a in r])
            arr[i].n_rays = len(r[0])
            arr[i].pixels = _lib.XkPixels(*[_ptr(a) for a in p])
            arr[i].n_pix = len(p[0])
            arr[i].out = _lib.XkField(*[_ptr(a) for a in o])
        self._arr = arr
        flags = 0 if graph else _lib.XK_BATCH_NO_GRAPH
        h = ctypes.c_void_p()
        rc = lib.xk_batch_create(self._ctx.handle, arr, len(solves), _path(path), flags,
                                 ctypes.byref(h))
        _lib.check(rc, self._ctx.handle)
        self._h = h
        self.n = len(solves)

    def run(self):
        st = _lib.XkBatchStats()
        _lib.check(_lib.load().xk_batch_run(self._h, ctypes.byref(st)), self._ctx.handle)
        self.stats = st.to_dict()
        return self.outputs

    def plan(self, i):
        pl = _lib.XkSolvePlan()
        _lib.check(_lib.load().xk_batch_solve_plan(self._h, i, ctypes.byref(pl)))
        return pl.to_dict()

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().xk_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(rays, pixels, out, ctx=None, budget_ms=3000.0, apply=True):
    """Tune the FP32-PR knobs on a device-resident problem (tensors with
    ``data_ptr()``); keeps the fastest settings on ``ctx`` when ``apply``."""
    ctx = _require_ctx(ctx)
    dp = ctypes.POINTER(ctypes.c_double)

    def cast(t):
        return ctypes.cast(ctypes.c_void_p(int(t.data_ptr())), dp)

    if isinstance(rays, dict):
        rays = [rays[k] for k in RAY_FIELDS]
    if isinstance(pixels, dict):
        pixels = [pixels[k] for k in PIXEL_FIELDS]
    res = _lib.XkTuneResult()
    rc = _lib.load().xk_autotune(ctx.handle, _lib.XkRays(*[cast(a) for a in rays]),
                                 int(rays[0].numel()), _lib.XkPixels(*[cast(a) for a in pixels]),
                                 int(pixels[0].numel()), _lib.XkField(*[cast(a) for a in out]),
                                 float(budget_ms), 1 if apply else 0, ctypes.byref(res))
    _lib.check(rc, ctx.handle)
    return res.to_dict()


def probe_pipes(ctx=None):
    """Peak rates of the FP32 FMA pipe (lane operations, an f32x2 FMA counting
    two) and of the MUFU unit (sin/cos results), per SM clock, measured on
    the device with every SM busy."""
    ctx = _require_ctx(ctx)
    res = _lib.XkPipePeaks()
    _lib.check(_lib.load().xk_probe_pipes(ctx.handle, ctypes.byref(res)), ctx.handle)
    return res.to_dict()


def _as_records(a, dtype):
    a = np.ascontiguousarray(a)
    if a.dtype != dtype:
        raise ValueError(f"expected dtype {dtype}")
    return a


def kirchhoff_gpu(ctx, rays, pixels):
    """gpu::kirchhoff::kirchhoff_gpu: GpuRay / GpuPixel records in, complex128
    arrays (es, ep) out, one entry per pixel."""
    if ctx is None:
        raise ValueError("ctx is required (use kirchhoff_auto for the shared context)")
    rays = _as_records(rays, GPU_RAY_DTYPE)
    pixels = _as_records(pixels, GPU_PIXEL_DTYPE)
    out = np.zeros((len(pixels), 4), dtype=np.float64)
    lib = _lib.load()
    rc = lib.xk_kirchhoff_gpu(ctx.handle, rays.ctypes.data_as(ctypes.POINTER(_lib.XkGpuRay)),
                              len(rays), pixels.ctypes.data_as(ctypes.POINTER(_lib.XkGpuPixel)),
                              len(pixels), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    _lib.check(rc, ctx.handle)
    return out[:, 0] + 1j * out[:, 1], out[:, 2] + 1j * out[:, 3]


def kirchhoff_auto(rays, pixels):
    """gpu::fallback::kirchhoff_auto on the shared context. No CPU fallback:
    raises XkError(XK_ERR_NO_DEVICE) without a device."""
    rays = _as_records(rays, GPU_RAY_DTYPE)
    pixels = _as_records(pixels, GPU_PIXEL_DTYPE)
    out = np.zeros((len(pixels), 4), dtype=np.float64)
    lib = _lib.load()
    rc = lib.xk_kirchhoff_auto(rays.ctypes.data_as(ctypes.POINTER(_lib.XkGpuRay)), len(rays),
                               pixels.ctypes.data_as(ctypes.POINTER(_lib.XkGpuPixel)), len(pixels),
                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    _lib.check(rc)
    return out[:, 0] + 1j * out[:, 1], out[:, 2] + 1j * out[:, 3]


from .waves import (WaveParams, prepare_wave, beam_to_diffraction_rays,  # noqa: E402
                    diffraction_from_beam)
from .fresnel import FresnelScreen, FresnelResult, fresnel_propagate  # noqa: E402
