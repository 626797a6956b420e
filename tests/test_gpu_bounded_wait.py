"""Device-side bounded waits run out, and the context stays usable.

The failure is made on the host: the "inject_stall" test hook makes the next
phase-reduced execution expect 16 bytes more on its first ray stage's barrier
than the stage's bulk copy delivers. The copy lands (nothing stays in
flight), the barrier can never complete, and the warp's bounded wait runs out
after "wait_limit" polls. The call must return XK_ERR_TIMEOUT, and the next
solve on the same context must be right: equal, bit for bit, to the same solve
on a context that never failed, and within 1e-4 of the oracle. The
"fresnel_stall" hook does the same for the tensor-core Fresnel product: its
first stage's barrier expects one arrival more than the producers make, so the
MMA issuer gives up before it issues anything. No GPU faults, traps or hangs:
every wait involved is bounded.
"""
import time

import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import _lib, synth

pytestmark = pytest.mark.gpu


def _solve(ctx, rays, pix):
    return xrt_rs.diffraction_integral(rays, pix, path="f32pr", ctx=ctx, return_stats=True)


def test_stalled_stage_times_out_and_context_recovers(oracle):
    rays, pix = synth.config0(seed=8)
    rl, pl = cases.as_lists(rays, pix)
    clean = xrt_rs.GpuContext.new(0)
    ref_out, _ = _solve(clean, rl, pl)
    clean.close()

    ctx = xrt_rs.GpuContext.new(0)
    try:
        ctx.set_option("wait_limit", 4096)
        ctx.set_option("inject_stall", 16)
        t0 = time.perf_counter()
        with pytest.raises(xrt_rs.XkError) as ei:
            _solve(ctx, rl, pl)
        dt = time.perf_counter() - t0
        assert ei.value.code == _lib.XK_ERR_TIMEOUT, str(ei.value)
        print(f"stalled solve returned XK_ERR_TIMEOUT after {dt * 1e3:.1f} ms: {ei.value}")
        # The hook armed one execution only; the default limit comes back.
        ctx.set_option("wait_limit", float(1 << 24))
        out, st = _solve(ctx, rl, pl)
        assert st["path"] == xrt_rs.XK_PATH_F32PR
        for a, b in zip(out, ref_out):
            assert np.array_equal(a, b)
        assert cases.rel_l2(out, oracle.kahan_f64(rl, pl)) < 1e-4
        # The FP64 path on the same context is unaffected as well.
        out64, _ = xrt_rs.diffraction_integral(rl, pl, path="f64", ctx=ctx, return_stats=True)
        assert cases.rel_l2(out64, oracle.kahan_f64(rl, pl)) < 1e-10
    finally:
        ctx.close()


def test_wait_limit_alone_keeps_results():
    """A lower (but sufficient) poll limit changes nothing when no stage stalls."""
    rays, pix = synth.config0(seed=9)
    rl, pl = cases.as_lists(rays, pix)
    ctx = xrt_rs.GpuContext.new(0)
    try:
        a, _ = _solve(ctx, rl, pl)
        ctx.set_option("wait_limit", float(1 << 20))
        b, _ = _solve(ctx, rl, pl)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    finally:
        ctx.close()


def test_option_validation():
    ctx = xrt_rs.GpuContext.new(0)
    try:
        for name, bad in (("wait_limit", 0), ("wait_limit", 1.5), ("wait_limit", 2.0 ** 32),
                          ("inject_stall", 8), ("inject_stall", 2048), ("inject_stall", -16),
                          ("fresnel_stall", 2), ("fresnel_stall", -1), ("fresnel_pair", 0.5)):
            with pytest.raises(xrt_rs.XkError) as ei:
                ctx.set_option(name, bad)
            assert ei.value.code == _lib.XK_ERR_INVALID
        ctx.set_option("inject_stall", 0)  # disarms
        ctx.set_option("fresnel_stall", 0)
    finally:
        ctx.close()


@pytest.mark.parametrize("nz", [64, 200])
def test_fresnel_stalled_stage_times_out_and_context_recovers(nz):
    """The tensor-core Fresnel product (one CTA per tile for nz = 64, CTA
    pairs for nz = 200): the "fresnel_stall" hook arms the first stage's
    barrier with one arrival more than the producers make, so the MMA issuer's
    bounded wait runs out before it issues anything. The call returns
    XK_ERR_TIMEOUT; the next call on the same context equals, bit for bit, the
    same call on a context that never failed."""
    rng = np.random.default_rng(nz)
    x, z = rng.normal(0, 0.05, 3000), rng.normal(0, 0.05, 3000)
    es = np.exp(1j * rng.uniform(-np.pi, np.pi, 3000))
    sc = xrt_rs.FresnelScreen(-0.2, 0.2, 150, -0.2, 0.2, nz)
    clean = xrt_rs.GpuContext.new(0)
    ref = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, ctx=clean).amplitude
    ref64 = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, path="f64", ctx=clean).amplitude
    clean.close()

    ctx = xrt_rs.GpuContext.new(0)
    try:
        ctx.set_option("wait_limit", 4096)
        ctx.set_option("fresnel_stall", 1)
        t0 = time.perf_counter()
        with pytest.raises(xrt_rs.XkError) as ei:
            xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, ctx=ctx)
        dt = time.perf_counter() - t0
        assert ei.value.code == _lib.XK_ERR_TIMEOUT, str(ei.value)
        print(f"stalled product returned XK_ERR_TIMEOUT after {dt * 1e3:.1f} ms: {ei.value}")
        ctx.set_option("wait_limit", float(1 << 24))
        res, st = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, ctx=ctx,
                                           return_stats=True)
        assert st["path"] == _lib.XK_PATH_SEPARABLE
        assert st["sweep"] == (1 if nz > 128 else 0)  # CTA pairs above 128 rows
        assert np.array_equal(res.amplitude, ref)
        assert np.linalg.norm(res.amplitude - ref64) / np.linalg.norm(ref64) < 1e-4
    finally:
        ctx.close()
