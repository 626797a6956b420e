"""2-D Fresnel propagation on the device (xk_fresnel_propagate).

XK_PATH_F64 is the reference's FP64 sum term for term and must match the
oracle's restatement of src/waves/fresnel.rs:53-106 to 1e-10; the
tensor-core separable product (XK_PATH_SEPARABLE) must match it to 1e-4
(relative L2 over the complex screen). Screen coordinates are exact."""
import numpy as np
import pytest

import xrt_rs
from xrt_rs import FresnelScreen

pytestmark = pytest.mark.gpu

F64_TOL = 1e-10
SEP_TOL = 1e-4


def rays(n, seed, spread=0.05):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, spread, n)
    z = rng.normal(0, spread, n)
    es = rng.uniform(0.2, 1.0, n) * np.exp(1j * rng.uniform(-np.pi, np.pi, n))
    return x, z, es


def oracle_field(oracle, x, z, es, energy, dist, sc):
    re, im = oracle.fresnel(x, z, es.real, es.imag, energy, dist, sc.x_min, sc.x_max, sc.nx,
                            sc.z_min, sc.z_max, sc.nz)
    return re + 1j * im


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def coords(lo, hi, n):
    return lo + (hi - lo) * np.arange(n, dtype=np.float64) / float(max(n - 1, 1))


CASES = [  # (n rays, screen, energy, dist)
    (3001, FresnelScreen(-0.3, 0.3, 37, -0.2, 0.25, 29), 10000.0, 1000.0),
    (777, FresnelScreen(-0.5, 0.5, 129, -0.5, 0.5, 129), 30000.0, 100.0),
    (64, FresnelScreen(-0.1, 0.1, 300, 0.0, 0.0, 1), 8000.0, 5000.0),
    (5000, FresnelScreen(0.2, 0.2, 1, -0.4, 0.4, 211), 1000.0, 20000.0),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_f64_matches_oracle(ctx, oracle, case):
    n, sc, energy, dist = CASES[case]
    x, z, es = rays(n, seed=case)
    res = xrt_rs.fresnel_propagate(x, z, es, energy, dist, sc, path="f64", ctx=ctx)
    ref = oracle_field(oracle, x, z, es, energy, dist, sc)
    assert res.amplitude.shape == (sc.nx * sc.nz,)
    assert rel(res.amplitude, ref) < F64_TOL
    assert np.array_equal(res.x_pixels, coords(sc.x_min, sc.x_max, sc.nx))
    assert np.array_equal(res.z_pixels, coords(sc.z_min, sc.z_max, sc.nz))


@pytest.mark.parametrize("case", range(len(CASES)))
def test_separable_matches_oracle(ctx, oracle, case):
    n, sc, energy, dist = CASES[case]
    x, z, es = rays(n, seed=case)
    res, st = xrt_rs.fresnel_propagate(x, z, es, energy, dist, sc, ctx=ctx, return_stats=True)
    ref = oracle_field(oracle, x, z, es, energy, dist, sc)
    err = rel(res.amplitude, ref)
    print(f"case {case}: separable rel L2 {err:.2e}, chunks {st['n_chunks']}, "
          f"tiles {st['n_tiles']} x splits {st['groups']}")
    assert st["path"] == xrt_rs._lib.XK_PATH_SEPARABLE
    assert err < SEP_TOL
    assert np.array_equal(res.x_pixels, coords(sc.x_min, sc.x_max, sc.nx))


def test_separable_many_segments_and_splits(ctx, oracle):
    """20011 rays on one output tile: K split over many CTAs, each running
    several accumulation segments through both tensor-memory accumulators."""
    x, z, es = rays(20011, seed=9)
    sc = FresnelScreen(-0.2, 0.2, 45, -0.2, 0.2, 33)
    res, st = xrt_rs.fresnel_propagate(x, z, es, 12000.0, 800.0, sc, ctx=ctx, return_stats=True)
    assert st["n_tiles"] == 1 and st["groups"] >= 8
    assert st["n_chunks"] == (20011 + 31) // 32  # ray blocks
    assert rel(res.amplitude, oracle_field(oracle, x, z, es, 12000.0, 800.0, sc)) < SEP_TOL


@pytest.mark.parametrize("path", ["f64", "separable"])
def test_single_point_source(ctx, path):
    """src/waves/fresnel.rs:127-145."""
    res = xrt_rs.fresnel_propagate([0.0], [0.0], [1.0 + 0j], 10000.0, 1000.0,
                                   FresnelScreen(-0.1, 0.1, 21, -0.1, 0.1, 21), path=path, ctx=ctx)
    assert len(res.amplitude) == 21 * 21
    a = np.abs(res.amplitude)
    assert a[10 * 21 + 10] >= a[0] - 1e-6
    assert np.allclose(a, 1.0, atol=1e-5)


@pytest.mark.parametrize("path", ["f64", "separable"])
def test_two_slit(ctx, path):
    """src/waves/fresnel.rs:147-165."""
    res = xrt_rs.fresnel_propagate([-0.01, 0.01], [0.0, 0.0], [1.0 + 0j, 1.0 + 0j], 10000.0,
                                   1000.0, FresnelScreen(-0.1, 0.1, 101, 0.0, 0.0, 1), path=path,
                                   ctx=ctx)
    inten = res.intensity()
    assert inten[50] > 0.0 and inten[60] > 0.0


@pytest.mark.parametrize("path", ["f64", "separable"])
def test_no_rays_and_zero_amplitudes(ctx, path):
    sc = FresnelScreen(-0.1, 0.1, 5, -0.1, 0.1, 4)
    res = xrt_rs.fresnel_propagate([], [], [], 10000.0, 1000.0, sc, path=path, ctx=ctx)
    assert np.all(res.amplitude == 0)
    res = xrt_rs.fresnel_propagate([0.0, 0.1], [0.0, 0.0], [0j, 0j], 10000.0, 1000.0, sc,
                                   path=path, ctx=ctx)
    assert np.all(res.amplitude == 0)


def test_empty_screen_and_bad_arguments(ctx):
    res = xrt_rs.fresnel_propagate([0.0], [0.0], [1 + 0j], 1e4, 1e3,
                                   FresnelScreen(-1, 1, 0, -1, 1, 5), ctx=ctx)
    assert res.amplitude.size == 0
    with pytest.raises(ValueError):
        xrt_rs.fresnel_propagate([0.0, 1.0], [0.0], [1 + 0j], 1e4, 1e3,
                                 FresnelScreen(-1, 1, 2, -1, 1, 2), ctx=ctx)
    with pytest.raises(ValueError):
        xrt_rs.fresnel_propagate([0.0], [0.0], [1 + 0j], 1e4, 1e3,
                                 FresnelScreen(-1, 1, 2, -1, 1, 2), path="f32", ctx=ctx)


@pytest.mark.parametrize("shape", [(300, 200), (129, 257), (64, 384)])
def test_cta_pair_tiles_match_single_cta_tiles(ctx, oracle, shape):
    """Screens of more than 128 rows run the product on CTA pairs (one tcgen05
    MMA over two SMs, 256 x 256 tiles, option "fresnel_pair" = 1, the
    default); "fresnel_pair" = 0 keeps one CTA per 128 x 256 tile. Both match
    the oracle and each other: bit for bit where both pad the screen to the same
    rows (and so split K the same way), else to the FP64 summation order of the
    K splits."""
    nx, nz = shape
    x, z, es = rays(3000, seed=31 + nx)
    sc = FresnelScreen(-0.3, 0.3, nx, -0.25, 0.2, nz)
    pair = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, ctx=ctx).amplitude
    ctx.set_option("fresnel_pair", 0)
    try:
        single = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, ctx=ctx).amplitude
    finally:
        ctx.set_option("fresnel_pair", 1)
    ref = oracle_field(oracle, x, z, es, 10000.0, 1000.0, sc)
    e_pair, e_single, e_both = rel(pair, ref), rel(single, ref), rel(pair, single)
    print(f"{nx}x{nz}: pair {e_pair:.2e}, single {e_single:.2e}, pair vs single {e_both:.2e}")
    assert e_pair < SEP_TOL and e_single < SEP_TOL
    assert e_both < 1e-6
    if (nz + 127) // 128 % 2 == 0:
        # Same padded rows, hence the same K splits: both kernels form the
        # same tiles and sums, bit for bit.
        assert np.array_equal(pair, single)


def test_separable_long_accumulation_against_f64(ctx):
    """Few K splits per output tile (a 1024x1024 screen has 64 tiles), so each
    CTA accumulates ~900 K blocks: the segmented FP64 drain keeps the product
    as accurate as in the short-K cases (checked against the GPU FP64 sum,
    itself pinned to the oracle above)."""
    x, z, es = rays(20_000, seed=11, spread=0.1)
    sc = FresnelScreen(-0.5, 0.5, 1024, -0.5, 0.5, 1024)
    sep, st = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, ctx=ctx, return_stats=True)
    ref = xrt_rs.fresnel_propagate(x, z, es, 10000.0, 1000.0, sc, path="f64", ctx=ctx)
    err = rel(sep.amplitude, ref.amplitude)
    print(f"long K: rel L2 {err:.2e}, tiles {st['n_tiles']} x splits {st['groups']}")
    assert st["groups"] <= 4
    assert err < 1e-5


def test_separable_routes_to_f64_beyond_the_cross_term_bound(ctx, oracle):
    """A screen of +-50 mm at 30 keV and 100 mm puts the FP32 cross term of the
    phase split beyond 2^21 turns: the call runs the FP64 sum instead and
    reports it."""
    rng = np.random.default_rng(21)
    x, z = rng.uniform(-1, 1, 300), rng.uniform(-1, 1, 300)
    es = np.exp(1j * rng.uniform(-np.pi, np.pi, 300))
    sc = FresnelScreen(-50.0, 50.0, 9, -50.0, 50.0, 7)
    res, st = xrt_rs.fresnel_propagate(x, z, es, 30000.0, 100.0, sc, ctx=ctx, return_stats=True)
    assert st["path"] == xrt_rs._lib.XK_PATH_F64
    assert rel(res.amplitude, oracle_field(oracle, x, z, es, 30000.0, 100.0, sc)) < F64_TOL


@pytest.mark.parametrize("geom", range(4))
@pytest.mark.parametrize("kind", ["one", "two", "row16", "row97"])
def test_closed_form_fields(ctx, geom, kind):
    """Both device paths against closed-form fields (point sources, a Talbot
    row summed as a geometric series): FP64 to 1e-10 (widened by the FP64
    rounding of the largest phase), the tensor-core product to 1e-4."""
    import fresnel_closed as F
    import test_fresnel_closed_form as T

    energy, dist, sc_t = T.GEOMS[geom]
    x, z, e, exact = T.sources(kind, energy, dist)
    sc = FresnelScreen(*sc_t)
    xp, zp = F.screen_coords(*sc_t)
    ref = exact(xp, zp)
    res = xrt_rs.fresnel_propagate(x, z, e, energy, dist, sc, path="f64", ctx=ctx)
    assert F.rel_l2(res.amplitude, ref) <= T.tol(F64_TOL, energy, dist, x, z, sc_t)
    res, st = xrt_rs.fresnel_propagate(x, z, e, energy, dist, sc, path="separable", ctx=ctx,
                                       return_stats=True)
    err = F.rel_l2(res.amplitude, ref)
    print(f"closed form {kind} E={energy} d={dist}: separable {err:.2e} path={st['path']}")
    assert err <= SEP_TOL
