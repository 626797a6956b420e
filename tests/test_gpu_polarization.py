"""One common polarization: every ray's (es, ep) a multiple of ray 0's.

Then Ep(p) = (ep_0 / es_0) Es(p) exactly in the reference's sum
(src/waves/diffraction.rs:67-117 is linear in (es, ep)), so the phase-reduced
kernels sum one amplitude column and scale it. This is the reference's own
benchmark (benches/diffraction.rs: es = 1, ep = 0) and beam_to_diffraction_rays
without amplitudes (src/waves/prepare_wave.rs:89-95). The detection tolerates
2^-24 of relative deviation per ray (below the FP32 rounding the kernel applies
to amplitudes anyway); anything more takes the two-column kernels.
"""
import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import synth

pytestmark = pytest.mark.gpu

PR_TOL = 1e-4


@pytest.fixture
def pol_ctx(ctx):
    yield ctx
    ctx.set_option("polarization", -1)


def with_amplitudes(es, ep, seed=5, n=20000):
    rays, pix = synth.config0(seed=seed)
    rays = dict(rays)
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, len(rays["x"]), n)
    rays = {k: np.asarray(v)[idx].copy() for k, v in rays.items()}
    es_v, ep_v = es(rays, rng), ep(rays, rng)
    rays["es_re"], rays["es_im"] = np.real(es_v).copy(), np.imag(es_v).copy()
    rays["ep_re"], rays["ep_im"] = np.real(ep_v).copy(), np.imag(ep_v).copy()
    return rays, pix


def gauss(rays, rng):
    return rays["es_re"] + 1j * rays["es_im"]


AMPS = {
    "reference_bench": (lambda r, g: np.ones(len(r["x"]), complex),
                        lambda r, g: np.zeros(len(r["x"]), complex)),
    "ep_tenth": (gauss, lambda r, g: 0.1 * gauss(r, g)),
    "complex_ratio": (gauss, lambda r, g: (0.3 - 0.7j) * gauss(r, g)),
    "es_zero": (lambda r, g: np.zeros(len(r["x"]), complex), gauss),
}


def run(ctx, rays, pix):
    return xrt_rs.diffraction_integral(*cases.as_lists(rays, pix), path="f32pr", ctx=ctx,
                                       return_stats=True)


@pytest.mark.parametrize("name", list(AMPS))
def test_one_polarization_matches_two_columns_and_oracle(pol_ctx, oracle, name):
    rays, pix = with_amplitudes(*AMPS[name])
    one, st1 = run(pol_ctx, rays, pix)
    assert st1["one_polarization"] == 1 and st1["path"] == xrt_rs.XK_PATH_F32PR
    pol_ctx.set_option("polarization", 0)
    two, st2 = run(pol_ctx, rays, pix)
    assert st2["one_polarization"] == 0
    if name != "es_zero":
        # The summed column is es. The folded one-column kernel sums it with
        # the FP32 operations of the two-column kernel's Es sum: bit for bit
        # the same Es. The unfolded one carries it in polar form (its phase
        # joins the pair's residual phase): another rounding of the same sum.
        es1 = one[0] + 1j * one[1]
        es2 = two[0] + 1j * two[1]
        if st1["folded"]:
            assert np.array_equal(one[0], two[0]) and np.array_equal(one[1], two[1])
        else:
            assert np.linalg.norm(es1 - es2) / np.linalg.norm(es2) < 5e-5
    ref = oracle.kahan_f64(*cases.as_lists(rays, pix))
    assert cases.rel_l2(one, ref) < PR_TOL
    assert cases.rel_l2(one, two) < (1e-6 if st1["folded"] else 5e-5)
    if name == "reference_bench":
        assert not np.any(one[2]) and not np.any(one[3])
    if name == "es_zero":
        assert not np.any(one[0]) and not np.any(one[1])


@pytest.mark.parametrize("dev", [0.0, 2e-8, 1e-6])
def test_detection_tolerance(pol_ctx, dev):
    """Per-ray deviations up to 2^-24 (relative) still count as one
    polarization; 1e-6 does not."""
    rng = np.random.default_rng(9)
    noise = 1.0 + dev * rng.choice([-1.0, 1.0], 20000)
    rays, pix = with_amplitudes(gauss, lambda r, g: 0.1 * gauss(r, g) * noise)
    out, st = run(pol_ctx, rays, pix)
    assert st["one_polarization"] == (1 if dev < 6e-8 else 0)


def test_general_amplitudes_take_two_columns(ctx):
    rays, pix = cases.random_case(3000, 700, seed=3)
    _, st = run(ctx, rays, pix)
    assert st["one_polarization"] == 0


def test_ray0_zero_amplitude_takes_two_columns(ctx):
    """Ray 0 is the pivot of the test: with (es_0, ep_0) = 0 nothing is
    concluded and both columns are summed."""
    rays, pix = with_amplitudes(gauss, lambda r, g: 0.1 * gauss(r, g))
    for k in ("es_re", "es_im", "ep_re", "ep_im"):
        rays[k][0] = 0.0
    _, st = run(ctx, rays, pix)
    assert st["one_polarization"] == 0


def test_config1_workload_is_one_polarization(ctx):
    rays, screen = synth.config1(seed=0, n_rays=1 << 14, grid=64)
    _, st = run(ctx, rays, screen)
    assert st["one_polarization"] == 1


def test_unfolded_polar_one_column_matches_two_columns(pol_ctx, oracle):
    """The far-field one-column kernel (unfolded, amplitude in polar form) on
    the 10 keV, 1 m aperture: within the tolerance of the extended-precision
    oracle, and within FP32-PR noise of the two-column kernel."""
    rays, screen = synth.config1(seed=4, n_rays=1 << 18, grid=256)
    one, st1 = run(pol_ctx, rays, screen)
    assert st1["one_polarization"] == 1 and st1["folded"] == 0
    pol_ctx.set_option("polarization", 0)
    two, st2 = run(pol_ctx, rays, screen)
    assert st2["one_polarization"] == 0
    assert cases.rel_l2(one, two) < 5e-5
    sub, idx = synth.subsample_screen(screen, 128, seed=2)
    exact = oracle.kahan_ld(*cases.as_lists(rays, sub))
    got = [o[idx] for o in one]
    assert cases.rel_l2(got, exact) < PR_TOL
    assert cases.rel_l2_intensity(got, exact) < PR_TOL
