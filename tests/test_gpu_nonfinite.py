"""Non-finite inputs (NaN, +-inf) on every entry point.

The reference sums them like any other value (src/waves/diffraction.rs:67-117
skips only path < 1e-30, which NaN never satisfies; src/waves/fresnel.rs:53-106
skips nothing), so NaN and inf reach the output. The FP32 phase-reduced
planner builds its frame and cell grid from the inputs' bounding boxes, so a
solve with any non-finite value takes the FP64 sum instead (routed reason 7),
and the separable Fresnel product does the same; the results then equal the
FP64 path's, NaN for NaN, and the oracle's pattern of non-finite outputs.
"""
import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import FresnelScreen, synth

pytestmark = pytest.mark.gpu

F64_TOL = 1e-10
NONFINITE_REASON = 7


def poisoned(field, index, value, target="rays", seed=2):
    rays, pix = synth.config0(seed=seed)
    rays = {k: np.array(v, dtype=np.float64) for k, v in rays.items()}
    pix = {k: np.array(v, dtype=np.float64) for k, v in pix.items()}
    (rays if target == "rays" else pix)[field][index] = value
    return rays, pix


def same_with_nan(a, b):
    return all(np.array_equal(x, y, equal_nan=True) for x, y in zip(a, b))


@pytest.mark.parametrize("target,field,index,value", [
    ("rays", "x", 17, np.nan),
    ("rays", "z", 0, np.inf),
    ("rays", "energy", 9999, np.nan),
    ("rays", "nz", 5, -np.inf),
    ("rays", "es_re", 123, np.nan),
    ("rays", "nl", 77, np.inf),
    ("pixels", "z", 100, np.inf),
    ("pixels", "x", 0, np.nan),
])
def test_solve_routes_to_f64_and_propagates(ctx, oracle, target, field, index, value):
    rays, pix = poisoned(field, index, value, target)
    lists = cases.as_lists(rays, pix)
    out, st = xrt_rs.diffraction_integral(*lists, path="f32pr", ctx=ctx, return_stats=True)
    assert st["path"] == xrt_rs.XK_PATH_F64
    assert st["routed_reason"] == NONFINITE_REASON
    assert xrt_rs.route_reason(NONFINITE_REASON) == "non-finite ray or screen values"
    f64 = xrt_rs.diffraction_integral(*lists, path="f64", ctx=ctx)
    assert same_with_nan(out, f64)
    ref = oracle.kahan_f64(*lists)
    for got, exp in zip(out, ref):
        assert np.array_equal(np.isfinite(got), np.isfinite(exp))
    finite = np.isfinite(ref[0]) & np.isfinite(ref[1]) & np.isfinite(ref[2]) & np.isfinite(ref[3])
    if target == "rays":
        assert not finite.any()  # one bad ray reaches every screen point
    else:
        assert finite.sum() == len(pix["x"]) - 1
        sel = [np.asarray(o)[finite] for o in out]
        exp = [np.asarray(o)[finite] for o in ref]
        assert cases.rel_l2(sel, exp) < F64_TOL


def test_finite_solve_is_not_routed(ctx):
    rays, pix = poisoned("x", 0, 0.0)
    _, st = xrt_rs.diffraction_integral(*cases.as_lists(rays, pix), path="f32pr", ctx=ctx,
                                        return_stats=True)
    assert st["path"] == xrt_rs.XK_PATH_F32PR and st["routed_reason"] == 0


def test_batch_isolates_a_nonfinite_solve(ctx):
    good = [(r, p) for r, p, _ in synth.config3(seed=4, count=4, ray_range=(300, 20000),
                                                 pix_range=(17, 3000))]
    bad = poisoned("y", 3, np.nan)
    solves = good[:2] + [bad] + good[2:]
    batch = xrt_rs.Batch(solves, path="f32pr", ctx=ctx)
    outs = batch.run()
    plan = batch.plan(2)
    assert plan["path"] == xrt_rs.XK_PATH_F64 and plan["routed_reason"] == NONFINITE_REASON
    for i, ((rays, pix), got) in enumerate(zip(solves, outs)):
        alone = xrt_rs.diffraction_integral(*cases.as_lists(rays, pix), path="f32pr", ctx=ctx)
        assert same_with_nan(got, alone), i
        if i != 2:
            assert all(np.isfinite(o).all() for o in got), i


def test_kirchhoff_gpu_records_nonfinite(ctx):
    rays, pix = poisoned("x", 4, np.nan)
    recs = np.zeros(len(rays["x"]), dtype=xrt_rs.GPU_RAY_DTYPE)
    for k in xrt_rs.GPU_RAY_DTYPE.names:
        recs[k] = rays[k]
    px = np.zeros(len(pix["x"]), dtype=xrt_rs.GPU_PIXEL_DTYPE)
    for k in "xyz":
        px[k] = pix[k]
    es, ep = xrt_rs.kirchhoff_gpu(ctx, recs, px)
    assert np.isnan(es).all() and np.isnan(ep).all()


@pytest.mark.parametrize("what", ["x", "es", "z_inf"])
def test_fresnel_nonfinite_takes_f64(ctx, oracle, what):
    rng = np.random.default_rng(11)
    n = 2000
    x = rng.normal(0, 0.05, n)
    z = rng.normal(0, 0.05, n)
    es = rng.uniform(0.2, 1.0, n) * np.exp(1j * rng.uniform(-np.pi, np.pi, n))
    if what == "x":
        x[7] = np.nan
    elif what == "es":
        es[0] = complex(np.nan, 0.0)
    else:
        z[1999] = np.inf
    sc = FresnelScreen(-0.2, 0.2, 33, -0.2, 0.2, 31)
    res, st = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, ctx=ctx, return_stats=True)
    assert st["path"] == xrt_rs.XK_PATH_F64
    f64 = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, path="f64", ctx=ctx)
    assert np.array_equal(res.amplitude, f64.amplitude, equal_nan=True)
    re, im = oracle.fresnel(x, z, es.real, es.imag, 10000.0, 1000.0, sc.x_min, sc.x_max, sc.nx,
                            sc.z_min, sc.z_max, sc.nz)
    assert np.array_equal(np.isfinite(res.amplitude), np.isfinite(re + 1j * im))
    assert not np.isfinite(res.amplitude).any()


def test_fresnel_all_zero_amplitudes_but_one_nan(ctx):
    """A zero-amplitude beam writes zeros without a sum, unless an amplitude
    is NaN: then the FP64 sum runs and the NaN reaches every screen point."""
    x = np.zeros(50)
    z = np.zeros(50)
    es = np.zeros(50, dtype=np.complex128)
    es[10] = complex(0.0, np.nan)
    sc = FresnelScreen(-0.1, 0.1, 9, -0.1, 0.1, 7)
    res, st = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, ctx=ctx, return_stats=True)
    assert st["path"] == xrt_rs.XK_PATH_F64
    assert np.isnan(res.amplitude).all()


AMP_RANGE_REASON = 8


@pytest.mark.parametrize("scale,routed", [(1e-35, True), (1e35, True), (1e-25, False),
                                          (1e25, False)])
def test_amplitude_range(ctx, oracle, scale, routed):
    """Amplitudes the FP32 sums cannot carry (beyond 1e30 or below 1e-30 in
    every component) take the FP64 sum; inside that range the phase-reduced
    result scales with them."""
    rays, pix = synth.config0(seed=6)
    rays = {k: np.array(v, dtype=np.float64) for k, v in rays.items()}
    base = xrt_rs.diffraction_integral(*cases.as_lists(rays, pix), path="f32pr", ctx=ctx)
    for k in ("es_re", "es_im", "ep_re", "ep_im"):
        rays[k] = rays[k] * scale
    lists = cases.as_lists(rays, pix)
    out, st = xrt_rs.diffraction_integral(*lists, path="f32pr", ctx=ctx, return_stats=True)
    if routed:
        assert st["path"] == xrt_rs.XK_PATH_F64 and st["routed_reason"] == AMP_RANGE_REASON
        ref = oracle.kahan_f64(*lists)
        assert cases.rel_l2(out, ref) < 1e-10
    else:
        assert st["path"] == xrt_rs.XK_PATH_F32PR
        scaled = [np.asarray(b) * scale for b in base]
        assert cases.rel_l2(out, scaled) < 1e-6

