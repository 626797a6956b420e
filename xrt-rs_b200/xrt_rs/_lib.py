"""ctypes binding of libxk.so (include/xk.h).

The library is the product: there is no pure-Python or CPU fallback. If
libxk.so has not been built, importing this module raises ImportError with
the build command.
"""
from __future__ import annotations

import ctypes
import os

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_DIR, "libxk.so")

XK_OK = 0
XK_ERR_NO_DEVICE = 1
XK_ERR_INVALID = 2
XK_ERR_OOM = 3
XK_ERR_BUDGET = 4
XK_ERR_CUDA = 5
XK_ERR_TIMEOUT = 6
XK_ERR_NOT_FOUND = 7
XK_ERR_CANCELLED = 8
XK_ERR_SHUTDOWN = 9

XK_PATH_F64 = 0
XK_PATH_F32PR = 1
XK_PATH_SEPARABLE = 2
XK_SERVE_SHORTEST_AGED = 0
XK_SERVE_EQUAL_SHARE = 1

_dp = ctypes.POINTER(ctypes.c_double)


class XkRays(ctypes.Structure):
    _fields_ = [(n, _dp) for n in ("x", "y", "z", "nx", "ny", "nz", "nl",
                                   "es_re", "es_im", "ep_re", "ep_im", "energy")]


class XkPixels(ctypes.Structure):
    _fields_ = [(n, _dp) for n in ("x", "y", "z")]


class XkField(ctypes.Structure):
    _fields_ = [(n, _dp) for n in ("es_re", "es_im", "ep_re", "ep_im")]


class XkGpuRay(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("x", "y", "z", "nx", "ny", "nz", "nl", "energy",
                                              "es_re", "es_im", "ep_re", "ep_im")]


class XkGpuPixel(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("x", "y", "z", "_pad")]


class XkStats(ctypes.Structure):
    _fields_ = [
        ("pairs", ctypes.c_double),
        ("gpu_ms", ctypes.c_double),
        ("wall_ms", ctypes.c_double),
        ("path", ctypes.c_int),
        ("kernels", ctypes.c_int),
        ("n_tiles", ctypes.c_int),
        ("n_chunks", ctypes.c_int),
        ("n_items", ctypes.c_longlong),
        ("phase_bound_rad", ctypes.c_double),
        ("h2d_bytes", ctypes.c_double),
        ("d2h_bytes", ctypes.c_double),
        ("main_kernel_ms", ctypes.c_double),
        ("groups", ctypes.c_int),
        ("routed_reason", ctypes.c_int),
        ("sweep", ctypes.c_int),
        ("one_polarization", ctypes.c_int),
        ("tuned", ctypes.c_int),
        ("folded", ctypes.c_int),
    ]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class XkSolve(ctypes.Structure):
    _fields_ = [("rays", XkRays), ("n_rays", ctypes.c_size_t), ("pixels", XkPixels),
                ("n_pix", ctypes.c_size_t), ("out", XkField)]


class XkBatchStats(ctypes.Structure):
    _fields_ = [
        ("pairs", ctypes.c_double), ("plan_ms", ctypes.c_double), ("exec_ms", ctypes.c_double),
        ("wall_ms", ctypes.c_double), ("n_solves", ctypes.c_int), ("routed_f64", ctypes.c_int),
        ("kernels", ctypes.c_int), ("graph", ctypes.c_int), ("n_items", ctypes.c_longlong),
    ]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class XkSolvePlan(ctypes.Structure):
    _fields_ = [("path", ctypes.c_int), ("routed_reason", ctypes.c_int), ("n_tiles", ctypes.c_int),
                ("n_chunks", ctypes.c_int), ("groups", ctypes.c_int), ("sweep", ctypes.c_int),
                ("phase_bound_rad", ctypes.c_double), ("one_polarization", ctypes.c_int),
                ("tuned", ctypes.c_int)]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class XkTuneResult(ctypes.Structure):
    _fields_ = [("default_ms", ctypes.c_double), ("best_ms", ctypes.c_double),
                ("phase_budget", ctypes.c_double), ("items_per_warp", ctypes.c_longlong),
                ("sweep", ctypes.c_int), ("trials", ctypes.c_int)]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class XkPipePeaks(ctypes.Structure):
    _fields_ = [("fma_lane_ops_per_clk_sm", ctypes.c_double),
                ("mufu_ops_per_clk_sm", ctypes.c_double), ("sm_clock_mhz", ctypes.c_double),
                ("fma_ms", ctypes.c_double), ("mufu_ms", ctypes.c_double),
                ("num_sms", ctypes.c_int)]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


XK_BATCH_DEVICE = 1
XK_BATCH_NO_GRAPH = 2


class XkServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_double), ("epoch_pairs", ctypes.c_double),
                ("max_active", ctypes.c_int), ("item_pairs", ctypes.c_double),
                ("inject_alloc_failure_every", ctypes.c_int), ("reserve_sms", ctypes.c_int),
                ("policy", ctypes.c_int), ("aging_ms", ctypes.c_double)]


class XkRequest(ctypes.Structure):
    _fields_ = [("rays", XkRays), ("n_rays", ctypes.c_size_t), ("rayset", ctypes.c_uint64),
                ("pixels", XkPixels), ("n_pix", ctypes.c_size_t), ("out", XkField),
                ("path", ctypes.c_int)]


class XkRequestStats(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("plan_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("path", ctypes.c_int), ("epochs", ctypes.c_int),
                ("status", ctypes.c_int)]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class XkServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong) for n in
                ("submitted", "completed", "failed", "epochs", "kernels", "pending", "active")] + \
               [(n, ctypes.c_double) for n in
                ("pairs_done", "used_bytes", "peak_bytes", "resident_ray_bytes",
                 "pairs_launched")]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}

class XkWaveParams(ctypes.Structure):
    _fields_ = [("center", ctypes.c_double * 3), ("dx", ctypes.c_double), ("dz", ctypes.c_double),
                ("nx", ctypes.c_size_t), ("nz", ctypes.c_size_t)]


class XkBeam(ctypes.Structure):
    _fields_ = [(n, _dp) for n in ("x", "y", "z", "a", "b", "c", "e",
                                   "es_re", "es_im", "ep_re", "ep_im")]


class XkRaysOut(ctypes.Structure):
    _fields_ = XkRays._fields_


class XkPixelsOut(ctypes.Structure):
    _fields_ = XkPixels._fields_


class XkFresnelScreen(ctypes.Structure):
    _fields_ = [("x_min", ctypes.c_double), ("x_max", ctypes.c_double), ("nx", ctypes.c_size_t),
                ("z_min", ctypes.c_double), ("z_max", ctypes.c_double), ("nz", ctypes.c_size_t)]


# Every entry point include/xk.h declares, with its ctypes signature.
_SIGNATURES = {
    "xk_init": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "xk_shared": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p)]),
    "xk_destroy": (None, [ctypes.c_void_p]),
    "xk_device_name": (ctypes.c_char_p, [ctypes.c_void_p]),
    "xk_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "xk_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "xk_version": (ctypes.c_char_p, []),
    "xk_route_reason": (ctypes.c_char_p, [ctypes.c_int]),
    "xk_set_option": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]),
    "xk_diffraction_integral": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.POINTER(XkRays), ctypes.c_size_t, ctypes.POINTER(XkPixels),
        ctypes.c_size_t, ctypes.POINTER(XkField), ctypes.c_int, ctypes.POINTER(XkStats)]),
    "xk_diffraction_integral_device": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.POINTER(XkRays), ctypes.c_size_t, ctypes.POINTER(XkPixels),
        ctypes.c_size_t, ctypes.POINTER(XkField), ctypes.c_int, ctypes.c_void_p,
        ctypes.POINTER(XkStats)]),
    "xk_kirchhoff_gpu": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.POINTER(XkGpuRay), ctypes.c_size_t, ctypes.POINTER(XkGpuPixel),
        ctypes.c_size_t, _dp]),
    "xk_diffraction_f64_noalloc": (ctypes.c_int, [
        ctypes.POINTER(XkRays), ctypes.c_size_t, ctypes.POINTER(XkPixels), ctypes.c_size_t,
        ctypes.POINTER(XkField), ctypes.c_void_p]),
    "xk_probe_pipes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XkPipePeaks)]),
    "xk_autotune": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.POINTER(XkRays), ctypes.c_size_t, ctypes.POINTER(XkPixels),
        ctypes.c_size_t, ctypes.POINTER(XkField), ctypes.c_double, ctypes.c_int,
        ctypes.POINTER(XkTuneResult)]),
    "xk_batch_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XkSolve), ctypes.c_size_t,
                                        ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "xk_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XkBatchStats)]),
    "xk_batch_solve_plan": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t,
                                            ctypes.POINTER(XkSolvePlan)]),
    "xk_batch_destroy": (None, [ctypes.c_void_p]),
    "xk_server_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XkServerOpts),
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "xk_server_upload_rays": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XkRays),
                                              ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)]),
    "xk_server_release_rays": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "xk_server_upload_beam": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.POINTER(XkBeam), ctypes.c_size_t, _dp,
        ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)]),
    "xk_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XkRequest),
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "xk_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double,
                                       ctypes.POINTER(XkRequestStats)]),
    "xk_server_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XkServerStats)]),
    "xk_server_destroy": (None, [ctypes.c_void_p]),
    "xk_prepare_wave": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XkWaveParams),
                                        ctypes.POINTER(XkPixelsOut)]),
    "xk_beam_to_rays": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.POINTER(XkBeam), ctypes.c_size_t, _dp,
        ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t, ctypes.POINTER(XkRaysOut)]),
    "xk_diffraction_beam": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.POINTER(XkBeam), ctypes.c_size_t, _dp,
        ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t, ctypes.POINTER(XkWaveParams),
        ctypes.POINTER(XkField), ctypes.c_int, ctypes.POINTER(XkStats)]),
    "xk_fresnel_propagate": (ctypes.c_int, [
        ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_size_t, ctypes.c_double, ctypes.c_double,
        ctypes.POINTER(XkFresnelScreen), _dp, _dp, _dp, _dp, ctypes.c_int,
        ctypes.POINTER(XkStats)]),
    "xk_kirchhoff_auto": (ctypes.c_int, [
        ctypes.POINTER(XkGpuRay), ctypes.c_size_t, ctypes.POINTER(XkGpuPixel), ctypes.c_size_t,
        _dp]),
}

_lib = None


def load():
    """Load libxk.so and attach signatures (cached)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python xrt-rs_b200/build.py`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_names():
    return sorted(_SIGNATURES)


class XkError(RuntimeError):
    """A non-zero status from the library."""

    def __init__(self, code: int, message: str):
        super().__init__(f"xk error {code}: {message}")
        self.code = code


def check(code: int, ctx=None):
    if code == XK_OK:
        return
    lib = load()
    msg = lib.xk_status_string(code).decode()
    if ctx:
        detail = lib.xk_last_error(ctx)
        if detail:
            msg = f"{msg}: {detail.decode()}"
    raise XkError(code, msg)
