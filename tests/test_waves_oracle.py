"""The screen-grid, beam-to-ray and Fresnel restatements in the oracle,
checked against the reference's own unit tests (no GPU):
src/waves/prepare_wave.rs:113-166, tests/pipeline.rs:167-191 and
src/waves/fresnel.rs:109-166."""
import numpy as np
import pytest

import cases


def test_prepare_wave_pixel_count(oracle):
    x, _, _ = oracle.prepare_wave([0.0, 1000.0, 0.0], 1.0, 1.0, 10, 10)
    assert len(x) == 100


def test_prepare_wave_center(oracle):
    x, y, z = oracle.prepare_wave([5.0, 1000.0, 3.0], 1.0, 1.0, 1, 1)
    assert len(x) == 1
    assert abs(x[0] - 5.0) < 1e-10 and abs(y[0] - 1000.0) < 1e-10 and abs(z[0] - 3.0) < 1e-10


def test_prepare_wave_grid_extent(oracle):
    x, _, _ = oracle.prepare_wave([0.0, 1000.0, 0.0], 5.0, 3.0, 11, 7)
    assert abs(x[0] + 5.0) < 1e-10
    assert abs(x[(11 - 1) * 7] - 5.0) < 1e-10


def test_prepare_wave_grid_properties(oracle):
    x, y, z = oracle.prepare_wave([10.0, 5000.0, -2.0], 3.0, 1.5, 21, 11)
    assert len(x) == 21 * 11
    assert np.all(np.abs(y - 5000.0) < 1e-10)
    assert abs(x.min() - 7.0) < 1e-10 and abs(x.max() - 13.0) < 1e-10
    assert abs(z.min() + 3.5) < 1e-10 and abs(z.max() + 0.5) < 1e-10


def test_prepare_wave_order_x_outer(oracle):
    x, _, z = oracle.prepare_wave([0.0, 0.0, 0.0], 1.0, 2.0, 3, 4)
    assert np.array_equal(x, np.repeat([-1.0, 0.0, 1.0], 4))
    assert np.array_equal(z, np.tile(np.linspace(-2.0, 2.0, 4), 3))


def test_beam_to_rays_basic(oracle):
    n = 3
    beam = {k: np.zeros(n) for k in ("x", "y", "z", "a", "b", "c", "e")}
    beam.update(es_re=np.zeros(n), es_im=np.zeros(n), ep_re=np.zeros(n), ep_im=np.zeros(n))
    beam["x"][0], beam["y"][0], beam["z"][0] = 1.0, 2.0, 3.0
    beam["b"][0] = 1.0
    beam["e"][0] = 10000.0
    beam["es_re"][0] = 1.0
    normals = np.tile([0.0, 0.0, 1.0], (n, 1))
    rays = oracle.beam_to_rays(beam, normals, [0])
    assert len(rays[0]) == 1
    assert abs(rays[0][0] - 1.0) < 1e-10 and abs(rays[11][0] - 10000.0) < 1e-10
    assert rays[6][0] == 0.0  # n . (0, 1, 0) with n = (0, 0, 1)


def test_beam_to_rays_without_amplitudes(oracle):
    beam, nrm, good = cases.beam_case(50, seed=1, amplitudes=False)
    r = oracle.beam_to_rays(beam, nrm, good)
    assert np.all(r[7] == 1.0) and np.all(r[8] == 0.0)
    assert np.all(r[9] == 0.0) and np.all(r[10] == 0.0)
    g = good.astype(np.int64)
    nl = nrm[g, 0] * beam["a"][g] + nrm[g, 1] * beam["b"][g] + nrm[g, 2] * beam["c"][g]
    assert np.array_equal(r[6], nl)


def test_beam_to_rays_rejects_out_of_range(oracle):
    beam, nrm, _ = cases.beam_case(10, seed=2)
    with pytest.raises(IndexError):
        oracle.beam_to_rays(beam, nrm, [10])


def test_fresnel_single_point_source(oracle):
    re, im = oracle.fresnel([0.0], [0.0], [1.0], [0.0], 10000.0, 1000.0,
                            -0.1, 0.1, 21, -0.1, 0.1, 21)
    assert len(re) == 21 * 21
    a = np.abs(re + 1j * im)
    assert a[10 * 21 + 10] >= a[0]


def test_fresnel_two_slit(oracle):
    re, im = oracle.fresnel([-0.01, 0.01], [0.0, 0.0], [1.0, 1.0], [0.0, 0.0], 10000.0, 1000.0,
                            -0.1, 0.1, 101, 0.0, 0.0, 1)
    inten = re ** 2 + im ** 2
    assert inten[50] > 0.0 and inten[60] > 0.0


def test_fresnel_matches_numpy_restatement(oracle):
    """The C restatement against a numpy evaluation of the same sum."""
    rng = np.random.default_rng(0)
    n = 40
    x, z = rng.normal(0, 0.05, n), rng.normal(0, 0.05, n)
    es = rng.normal(size=n) + 1j * rng.normal(size=n)
    re, im = oracle.fresnel(x, z, es.real, es.imag, 8000.0, 500.0, -0.2, 0.3, 7, -0.1, 0.1, 5)
    k = 8000.0 / 1973.2697177417986 * 1e7
    xs = -0.2 + 0.5 * np.arange(7) / 6.0
    zs = -0.1 + 0.2 * np.arange(5) / 4.0
    zp, xp = np.meshgrid(zs, xs, indexing="ij")
    r2 = (xp.reshape(-1, 1) - x) ** 2 + (zp.reshape(-1, 1) - z) ** 2
    ref = (es * np.exp(1j * (k / 1000.0) * r2)).sum(axis=1)
    got = re + 1j * im
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-9
