"""Screen grid and beam-to-ray producers on the device (xk_prepare_wave,
xk_beam_to_rays, xk_diffraction_beam).

Both producers are exact arithmetic in the reference's operation order, so
they must equal the oracle's restatement bit for bit; the chained solve must
equal xk_diffraction_integral on those rays and that screen bit for bit."""
import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import WaveParams

pytestmark = pytest.mark.gpu

GRIDS = [((0.0, 1000.0, 0.0), 1.0, 1.0, 10, 10), ((5.0, 1000.0, 3.0), 1.0, 1.0, 1, 1),
         ((10.0, 5000.0, -2.0), 3.0, 1.5, 21, 11), ((0.1, 2000.0, -0.3), 0.7, 0.2, 1, 333),
         ((-1.0, 800.0, 0.25), 0.05, 2.5, 517, 1), ((0.0, 1000.0, 0.0), 0.5, 0.5, 1000, 701)]


@pytest.mark.parametrize("grid", GRIDS)
def test_prepare_wave_bitwise(ctx, oracle, grid):
    c, dx, dz, nx, nz = grid
    got = xrt_rs.prepare_wave(WaveParams(c, dx, dz, nx, nz), ctx=ctx)
    ref = oracle.prepare_wave(c, dx, dz, nx, nz)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_prepare_wave_empty(ctx):
    x, y, z = xrt_rs.prepare_wave(WaveParams((0, 0, 0), 1.0, 1.0, 0, 5), ctx=ctx)
    assert len(x) == len(y) == len(z) == 0


@pytest.mark.parametrize("amplitudes", [True, False])
def test_beam_to_rays_bitwise(ctx, oracle, amplitudes):
    beam, nrm, good = cases.beam_case(20_011, seed=5, amplitudes=amplitudes)
    got = xrt_rs.beam_to_diffraction_rays(beam, nrm, good, ctx=ctx)
    ref = oracle.beam_to_rays(beam, nrm, good)
    for k, b in zip(xrt_rs.RAY_FIELDS, ref):
        assert np.array_equal(got[k], b), k


def test_beam_to_rays_rejects_bad_index(ctx):
    beam, nrm, _ = cases.beam_case(100, seed=6)
    with pytest.raises(xrt_rs.XkError) as ei:
        xrt_rs.beam_to_diffraction_rays(beam, nrm, [3, 100], ctx=ctx)
    assert ei.value.code == xrt_rs._lib.XK_ERR_INVALID
    with pytest.raises(ValueError):
        xrt_rs.beam_to_diffraction_rays({k: v for k, v in beam.items() if k != "ep_im"}, nrm,
                                        [0], ctx=ctx)


@pytest.mark.parametrize("path", ["f64", "f32pr"])
def test_diffraction_from_beam_equals_two_step(ctx, oracle, path):
    """tests/pipeline.rs:13-54 shape: beam after a mirror, screen at y = 2000."""
    beam, nrm, good = cases.beam_case(3000, seed=7)
    params = WaveParams((0.0, 2000.0, 0.0), 0.3, 0.3, 33, 31)
    got, st = xrt_rs.diffraction_from_beam(beam, nrm, good, params, path=path, ctx=ctx,
                                           return_stats=True)
    rays = dict(zip(xrt_rs.RAY_FIELDS, oracle.beam_to_rays(beam, nrm, good)))
    pix = dict(zip(xrt_rs.PIXEL_FIELDS, oracle.prepare_wave(params.center, params.dx, params.dz,
                                                            params.nx, params.nz)))
    two = xrt_rs.diffraction_integral(rays, pix, path=path, ctx=ctx)
    for a, b in zip(got, two):
        assert np.array_equal(a, b)
    assert st["path"] == xrt_rs._path(path)
    if path == "f64":
        ref = oracle.kahan_f64(*cases.as_lists(rays, pix))
        assert cases.rel_l2(got, ref) < 1e-10
    else:
        ref = oracle.kahan_ld(*cases.as_lists(rays, pix))
        assert cases.rel_l2(got, ref) < 1e-4
    es = np.abs(got[0] + 1j * got[1])
    assert es[(33 // 2) * 31 + 31 // 2] > 0.0  # non-zero at the screen centre (pipeline.rs:47-53)


def test_diffraction_from_beam_no_good_rays(ctx):
    beam, nrm, _ = cases.beam_case(10, seed=8)
    out = xrt_rs.diffraction_from_beam(beam, nrm, [], WaveParams((0, 2000.0, 0), 0.1, 0.1, 4, 4),
                                       ctx=ctx)
    assert all(np.all(o == 0.0) for o in out)
