"""Calls from several host threads at once.

The reference calls diffraction_integral from inside Rayon and keeps one
process-wide GpuContext (src/gpu/context.rs:28-31), so the library must accept
concurrent calls: on the shared context they serialize on its lock, on private
contexts they run side by side. ctypes releases the GIL for the duration of
each foreign call, so these threads really are inside the library together.
Every result must equal, bit for bit, the same call made alone.
"""
import threading

import numpy as np
import pytest

import cases
import xrt_rs

pytestmark = pytest.mark.gpu

JOBS = [(1500 + 97 * i, 300 + 41 * i, seed, path)
        for i, (seed, path) in enumerate([(1, "f32pr"), (2, "f64"), (3, "f32pr"), (4, "f32pr"),
                                          (5, "f64"), (6, "f32pr"), (7, "f32pr"), (8, "f64")])]


def _solve(job, ctx):
    n, m, seed, path = job
    rays, pix = cases.random_case(n, m, seed=seed)
    return xrt_rs.diffraction_integral(*cases.as_lists(rays, pix), path=path, ctx=ctx)


def _run_threads(fn, n_threads):
    results, errors = {}, []

    def worker(k):
        try:
            for i, job in enumerate(JOBS):
                if i % n_threads == k:
                    results[i] = fn(job, k)
        except Exception as e:  # reported on the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(n_threads)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
    return results


def test_threads_on_the_shared_context():
    shared = xrt_rs.GpuContext.shared()
    alone = [_solve(job, shared) for job in JOBS]
    got = _run_threads(lambda job, k: _solve(job, shared), 4)
    for i, a in enumerate(alone):
        for x, y in zip(a, got[i]):
            assert np.array_equal(x, y), i


def test_threads_on_private_contexts(ctx):
    alone = [_solve(job, ctx) for job in JOBS]
    ctxs = [xrt_rs.GpuContext.new(0) for _ in range(4)]
    try:
        got = _run_threads(lambda job, k: _solve(job, ctxs[k]), 4)
    finally:
        for c in ctxs:
            c.close()
    for i, a in enumerate(alone):
        for x, y in zip(a, got[i]):
            assert np.array_equal(x, y), i


def test_kirchhoff_auto_from_threads():
    """gpu::fallback::kirchhoff_auto on the shared context from four threads."""
    recs_pix = []
    for seed in range(8):
        rays, pix = cases.random_case(800 + 31 * seed, 150 + 7 * seed, seed=20 + seed)
        recs = np.zeros(len(rays["x"]), dtype=xrt_rs.GPU_RAY_DTYPE)
        for k in xrt_rs.GPU_RAY_DTYPE.names:
            recs[k] = rays[k]
        px = np.zeros(len(pix["x"]), dtype=xrt_rs.GPU_PIXEL_DTYPE)
        for k in "xyz":
            px[k] = pix[k]
        recs_pix.append((recs, px))
    alone = [xrt_rs.kirchhoff_auto(r, p) for r, p in recs_pix]
    results, errors = {}, []

    def worker(k):
        try:
            for i in range(k, len(recs_pix), 4):
                results[i] = xrt_rs.kirchhoff_auto(*recs_pix[i])
        except Exception as e:
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for i, (es, ep) in enumerate(alone):
        assert np.array_equal(es, results[i][0]) and np.array_equal(ep, results[i][1]), i
