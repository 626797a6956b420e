"""Continuous-batching server (xk_server_*), Python side.

    srv = Server(ctx, hbm_budget_bytes=120e9)
    h = srv.upload_rays(rays)                 # resident ray set, reused by many screens
    t = srv.submit(pixels, rays=None, rayset=h)   # returns at once
    es_re, es_im, ep_re, ep_im = srv.wait(t)   # blocks; srv.last_stats has latencies

Every request keeps its numpy buffers alive until it has been waited for.
With ``log=path`` every waited-for request appends one JSON line (ticket,
status, pairs, queue/plan/run/total ms, epochs, path) followed by the
server's counters (queue depth, active requests, bytes admitted).
"""
from __future__ import annotations

import ctypes
import json
import time

import numpy as np

from . import _lib
from . import (PIXEL_FIELDS, RAY_FIELDS, XkError, _check_lengths, _f64, _path, _ptr,
               _require_ctx)


class Server:
    def __init__(self, ctx=None, hbm_budget_bytes=0.0, epoch_pairs=0.0, max_active=0,
                 item_pairs=0.0, inject_alloc_failure_every=0, reserve_sms=0, log=None,
                 policy=0, aging_ms=0.0):
        self._ctx = _require_ctx(ctx)
        self._log = open(log, "a") if log else None
        opts = _lib.XkServerOpts(float(hbm_budget_bytes), float(epoch_pairs), int(max_active),
                                 float(item_pairs), int(inject_alloc_failure_every),
                                 int(reserve_sms), int(policy), float(aging_ms))
        h = ctypes.c_void_p()
        _lib.check(_lib.load().xk_server_create(self._ctx.handle, ctypes.byref(opts),
                                                ctypes.byref(h)), self._ctx.handle)
        self._h = h
        self._live = {}      # ticket -> (buffers kept alive, outputs)
        self._sets = {}      # rayset -> kept buffers
        self.last_stats = None

    @staticmethod
    def _rays(rays):
        if isinstance(rays, dict):
            rays = [rays[k] for k in RAY_FIELDS]
        r = [_f64(a) for a in rays]
        _check_lengths([("ray_" + n, len(a)) for n, a in zip(RAY_FIELDS, r)])
        return r

    def upload_rays(self, rays) -> int:
        r = self._rays(rays)
        h = ctypes.c_uint64()
        xr = _lib.XkRays(*[_ptr(a) for a in r])
        _lib.check(_lib.load().xk_server_upload_rays(self._h, ctypes.byref(xr), len(r[0]),
                                                     ctypes.byref(h)))
        self._sets[h.value] = r
        return h.value

    def upload_beam(self, beam, normals, good) -> int:
        """A resident ray set made on the device from a beam's columns
        (beam_to_diffraction_rays of ``good``; arguments as
        ``xrt_rs.beam_to_diffraction_rays``). Returns its handle."""
        from .waves import _beam_args
        xb, n, nrm, g, keep = _beam_args(beam, normals, good)
        h = ctypes.c_uint64()
        gp = g.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t))
        _lib.check(_lib.load().xk_server_upload_beam(self._h, ctypes.byref(xb), n, _ptr(nrm), gp,
                                                     len(g), ctypes.byref(h)))
        del keep
        return h.value

    def release_rays(self, handle: int):
        _lib.check(_lib.load().xk_server_release_rays(self._h, handle))
        self._sets.pop(handle, None)

    def submit(self, pixels, rays=None, rayset=0, path="f32pr") -> int:
        if isinstance(pixels, dict):
            pixels = [pixels[k] for k in PIXEL_FIELDS]
        p = [_f64(a) for a in pixels]
        _check_lengths([("pix_" + n, len(a)) for n, a in zip(PIXEL_FIELDS, p)])
        m = len(p[0])
        out = [np.zeros(m, dtype=np.float64) for _ in range(4)]
        keep = list(p) + out
        req = _lib.XkRequest()
        if rays is not None:
            r = self._rays(rays)
            keep += r
            req.rays = _lib.XkRays(*[_ptr(a) for a in r])
            req.n_rays = len(r[0])
        req.rayset = int(rayset)
        req.pixels = _lib.XkPixels(*[_ptr(a) for a in p])
        req.n_pix = m
        req.out = _lib.XkField(*[_ptr(a) for a in out])
        req.path = _path(path)
        t = ctypes.c_uint64()
        _lib.check(_lib.load().xk_server_submit(self._h, ctypes.byref(req), ctypes.byref(t)))
        self._live[t.value] = (keep, tuple(out))
        return t.value

    def wait(self, ticket: int, timeout_ms: float = -1.0):
        st = _lib.XkRequestStats()
        rc = _lib.load().xk_server_wait(self._h, ticket, float(timeout_ms), ctypes.byref(st))
        if rc == _lib.XK_ERR_TIMEOUT and timeout_ms >= 0 and st.total_ms == 0.0:
            raise XkError(rc, "wait timed out; the request is still running")
        keep, out = self._live.pop(ticket)
        self.last_stats = st.to_dict()
        if self._log is not None:
            rec = {"t": time.time(), "ticket": ticket, "rc": rc, **self.last_stats}
            srv = self.stats()
            rec.update({"queue_depth": srv["pending"], "active": srv["active"],
                        "admitted_bytes": srv["used_bytes"]})
            self._log.write(json.dumps(rec) + "\n")
            self._log.flush()
        _lib.check(rc)
        return out

    def stats(self):
        st = _lib.XkServerStats()
        _lib.check(_lib.load().xk_server_get_stats(self._h, ctypes.byref(st)))
        return st.to_dict()

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().xk_server_destroy(self._h)
            self._h = None
        self._live.clear()
        self._sets.clear()
        if getattr(self, "_log", None) is not None:
            self._log.close()
            self._log = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
