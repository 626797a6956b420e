"""The CPU oracle pinned against the reference's golden vectors (no GPU).

The reference fixture (validation/fixtures/diffraction_ref.json, copied to
tests/golden/) is checked at abs 1e-10 per component, the bar of
tests/golden_diffraction.rs:119-188 and validation/test_diffraction.py:36-59.
The reference's qualitative unit tests (src/waves/diffraction.rs:119-398) are
restated on the oracle so the inputs the GPU tests reuse are known-good.
"""
import numpy as np
import pytest

import cases

COMPS = ("es_re", "es_im", "ep_re", "ep_im")


def _golden_io(case):
    rays = [case["rays"][k] for k in cases.RAY_FIELDS]
    pix = [case["pixels"][k] for k in cases.PIXEL_FIELDS]
    return rays, pix


def test_kahan_oracle_matches_reference_fixture(oracle, golden_case):
    rays, pix = _golden_io(golden_case)
    out = oracle.kahan_f64(rays, pix)
    for i, exp in enumerate(golden_case["expected"]):
        for c, name in enumerate(COMPS):
            assert abs(out[c][i] - exp[name]) < 1e-10, (i, name, out[c][i], exp[name])


def test_plain_oracle_matches_reference_fixture(oracle, golden_case):
    rays, pix = _golden_io(golden_case)
    out = oracle.plain_f64(rays, pix)
    for i, exp in enumerate(golden_case["expected"]):
        for c, name in enumerate(COMPS):
            assert abs(out[c][i] - exp[name]) < 1e-10


def test_wgsl_restatement_within_reference_gpu_tolerance(oracle, golden_case):
    """tests/golden_gpu_kirchhoff.rs:103-145: GPU vs CPU at rel < 1e-3 per pixel."""
    r = golden_case["rays"]
    gpu_rays = [np.asarray(r[k], dtype=np.float32) for k in
                ("x", "y", "z", "nx", "ny", "nz", "nl", "energy", "es_re", "es_im", "ep_re", "ep_im")]
    pix = [np.asarray(golden_case["pixels"][k], dtype=np.float32) for k in "xyz"]
    out = oracle.wgsl_f32(gpu_rays, pix)
    ref_rays = [np.asarray(r[k], dtype=np.float32).astype(np.float64) for k in cases.RAY_FIELDS]
    ref = oracle.plain_f64(ref_rays, [p.astype(np.float64) for p in pix])
    for i in range(3):
        g = out[0][i] + 1j * out[1][i]
        c = ref[0][i] + 1j * ref[1][i]
        assert abs(g) > 1e-10
        assert abs(g - c) / abs(c) < 1e-3


def test_single_ray(oracle):
    rays, pix = cases.as_lists(*cases.single_ray_single_pixel())
    out = oracle.kahan_f64(rays, pix)
    assert abs(out[0][0] + 1j * out[1][0]) > 0.0
    assert abs(out[2][0] + 1j * out[3][0]) < 1e-30


def test_centre_brighter(oracle):
    rays, pix = cases.as_lists(*cases.parallel_pixels())
    out = oracle.kahan_f64(rays, pix)
    inten = out[0] ** 2 + out[1] ** 2
    assert inten[25] > inten[0]


def test_coincident_ray_skipped(oracle):
    rays, pix = cases.as_lists(*cases.ray_at_pixel())
    out = oracle.kahan_f64(rays, pix)
    assert all(abs(o[0]) < 1e-30 for o in out)


def test_kahan_stability(oracle):
    rays, pix = cases.as_lists(*cases.kahan_stability())
    big = oracle.kahan_f64(rays, pix)
    i = np.arange(100)
    small_rays = cases.rays_from((i - 50.0) * 0.001, es=0.01 + 0j)
    small = oracle.kahan_f64(*cases.as_lists(small_rays, cases.pixels_from([0.0], 0.0, 100.0)))
    a = abs(big[0][0] + 1j * big[1][0])
    b = abs(small[0][0] + 1j * small[1][0])
    assert np.isfinite(a) and a > 0
    assert 0.01 < a / b < 100.0


def test_large_ray_count(oracle):
    rays, pix = cases.as_lists(*cases.large_ray_count())
    out = oracle.kahan_f64(rays, pix)
    e = np.abs(out[0] + 1j * out[1])
    assert e[0] > 0.5 * e[1]


def test_polychromatic_finite(oracle):
    rays, pix = cases.as_lists(*cases.polychromatic())
    out = oracle.kahan_f64(rays, pix)
    assert np.isfinite(out[0][0]) and abs(out[0][0] + 1j * out[1][0]) > 0


def test_symmetry(oracle):
    rays, pix = cases.as_lists(*cases.symmetry())
    out = oracle.kahan_f64(rays, pix)
    e = np.abs(out[0] + 1j * out[1])
    assert abs(e[0] - e[1]) < 1e-10


def test_f64_sin_large_argument():
    """src/waves/diffraction.rs:287-305: f64 sin keeps precision at 2*pi*1e9."""
    base = 2.0 * np.pi * 1e9
    assert abs(np.sin(base + 0.001) - np.sin(0.001)) < 1e-6


def test_thread_count_does_not_change_results(oracle):
    rays, pix = cases.as_lists(*cases.random_case(300, 37, seed=3))
    a = oracle.kahan_f64(rays, pix, threads=1)
    b = oracle.kahan_f64(rays, pix, threads=4)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_empty_rays_give_zero(oracle):
    out = oracle.kahan_f64([[]] * 12, [[0.0], [0.0], [1000.0]])
    assert all(o[0] == 0.0 for o in out)


def test_extended_phase_oracle_measures_fp64_phase_rounding(oracle):
    """oracle_kahan_ld differs from the FP64 formula only by FP64's rounding of
    k*|p - r|: ~1e-6 at 10 keV and 1 m (5e10 rad), ~1e-4 at 24 keV and 8 m."""
    from xrt_rs import synth
    rays, pix = synth.config0(seed=0)
    rl, pl = cases.as_lists(rays, pix)
    d = cases.rel_l2(oracle.kahan_f64(rl, pl), oracle.kahan_ld(rl, pl))
    assert 1e-8 < d < 1e-5
    far, fpix, _ = synth.config3(seed=0, count=2, ray_range=(300, 30000), pix_range=(17, 4000))[1]
    rl, pl = cases.as_lists(far, fpix)
    d_far = cases.rel_l2(oracle.kahan_f64(rl, pl), oracle.kahan_ld(rl, pl))
    assert d_far > 10 * d
