"""GPU parity: libxk.so against the CPU oracle on the same seeded inputs.

Tolerances:
  XK_PATH_F64   rel L2 <= 1e-10 on the complex field (and abs 1e-10 per
                component on the reference fixture);
  XK_PATH_F32PR rel L2 <= 1e-4 on the complex field and on |E|^2.
"""
import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import synth

pytestmark = pytest.mark.gpu

F64_TOL = 1e-10
PR_TOL = 1e-4
COMPS = ("es_re", "es_im", "ep_re", "ep_im")


def run(ctx, rays, pix, path):
    r, p = cases.as_lists(rays, pix)
    out, st = xrt_rs.diffraction_integral(r, p, path=path, ctx=ctx, return_stats=True)
    return out, st


def oracle_run(oracle, rays, pix):
    return oracle.kahan_f64(*cases.as_lists(rays, pix))


def test_fixture_f64_abs_1e10(ctx, golden_case):
    rays = [golden_case["rays"][k] for k in cases.RAY_FIELDS]
    pix = [golden_case["pixels"][k] for k in cases.PIXEL_FIELDS]
    out = xrt_rs.diffraction_integral_rs(*rays, *pix)
    for i, exp in enumerate(golden_case["expected"]):
        for c, name in enumerate(COMPS):
            assert abs(out[c][i] - exp[name]) < 1e-10, (i, name)


def test_fixture_f32pr(ctx, golden_case):
    rays = [golden_case["rays"][k] for k in cases.RAY_FIELDS]
    pix = [golden_case["pixels"][k] for k in cases.PIXEL_FIELDS]
    out = xrt_rs.diffraction_integral_rs(*rays, *pix, path="f32pr")
    exp = [np.array([e[c] for e in golden_case["expected"]]) for c in COMPS]
    assert cases.rel_l2(out, exp) < PR_TOL


@pytest.mark.parametrize("builder", [
    cases.single_ray_single_pixel, cases.parallel_pixels, cases.ray_at_pixel,
    cases.kahan_stability, cases.polychromatic, cases.symmetry, cases.gpu_short_distance,
    cases.gpu_extreme_distance])
def test_reference_unit_cases_f64(ctx, oracle, builder):
    rays, pix = builder()
    out, st = run(ctx, rays, pix, "f64")
    ref = oracle_run(oracle, rays, pix)
    if np.linalg.norm(np.concatenate(cases.field_c(ref))) == 0:
        assert np.all(np.concatenate(out) == 0)
    else:
        assert cases.rel_l2(out, ref) < F64_TOL


@pytest.mark.parametrize("builder", [
    cases.single_ray_single_pixel, cases.parallel_pixels, cases.kahan_stability,
    cases.large_ray_count, cases.symmetry, cases.gpu_extreme_distance])
def test_reference_unit_cases_f32pr(ctx, oracle, builder):
    rays, pix = builder()
    out, st = run(ctx, rays, pix, "f32pr")
    ref = oracle_run(oracle, rays, pix)
    assert cases.rel_l2(out, ref) < PR_TOL, st


def test_polychromatic_routes_to_f64(ctx, oracle):
    rays, pix = cases.polychromatic()
    out, st = run(ctx, rays, pix, "f32pr")
    assert st["path"] == xrt_rs.XK_PATH_F64
    assert cases.rel_l2(out, oracle_run(oracle, rays, pix)) < F64_TOL


def test_coincident_ray_routes_to_f64_and_is_skipped(ctx):
    rays, pix = cases.ray_at_pixel()
    out, st = run(ctx, rays, pix, "f32pr")
    assert st["path"] == xrt_rs.XK_PATH_F64
    assert all(o[0] == 0.0 for o in out)


@pytest.mark.parametrize("n_rays,n_pix", cases.BENCH_SIZES)
def test_bench_sizes(ctx, oracle, n_rays, n_pix):
    rays, pix = cases.bench_case(n_rays, n_pix)
    ref = oracle_run(oracle, rays, pix)
    out64, _ = run(ctx, rays, pix, "f64")
    assert cases.rel_l2(out64, ref) < F64_TOL
    out32, _ = run(ctx, rays, pix, "f32pr")
    assert cases.rel_l2(out32, ref) < PR_TOL


@pytest.mark.parametrize("n_rays", [1, 2, 3, 7, 33, 65, 129])
@pytest.mark.parametrize("n_pix", [1, 5, 9, 31, 257])
def test_odd_sizes(ctx, oracle, n_rays, n_pix):
    rays, pix = cases.random_case(n_rays, n_pix, seed=n_rays * 1000 + n_pix)
    ref = oracle_run(oracle, rays, pix)
    out64, _ = run(ctx, rays, pix, "f64")
    assert cases.rel_l2(out64, ref) < F64_TOL
    out32, _ = run(ctx, rays, pix, "f32pr")
    assert cases.rel_l2(out32, ref) < PR_TOL


def test_exhaustive_tiny_sizes(ctx, oracle):
    """Every size of 1-7 rays x 1-9 screen points on both paths: the smallest
    cases hit every partial warp, stage and tile edge."""
    for n_rays in range(1, 8):
        for n_pix in range(1, 10):
            rays, pix = cases.random_case(n_rays, n_pix, seed=100 * n_rays + n_pix)
            ref = oracle_run(oracle, rays, pix)
            out64, _ = run(ctx, rays, pix, "f64")
            assert cases.rel_l2(out64, ref) < F64_TOL, (n_rays, n_pix)
            out32, _ = run(ctx, rays, pix, "f32pr")
            assert cases.rel_l2(out32, ref) < PR_TOL, (n_rays, n_pix)


def test_general_normals(ctx, oracle):
    rays, pix = cases.random_case(3000, 700, seed=11, general_normals=True)
    ref = oracle_run(oracle, rays, pix)
    out64, _ = run(ctx, rays, pix, "f64")
    assert cases.rel_l2(out64, ref) < F64_TOL
    out32, _ = run(ctx, rays, pix, "f32pr")
    assert cases.rel_l2(out32, ref) < PR_TOL


def test_empty_inputs(ctx):
    out, _ = run(ctx, cases.rays_from([]), cases.pixels_from([0.0, 1.0], 0.0, 1000.0), "f64")
    assert all(np.all(o == 0) for o in out)
    out, _ = run(ctx, cases.rays_from([]), cases.pixels_from([0.0, 1.0], 0.0, 1000.0), "f32pr")
    assert all(np.all(o == 0) for o in out)
    out, _ = run(ctx, cases.rays_from([0.0]), cases.pixels_from([], 0.0, 1000.0), "f32pr")
    assert all(len(o) == 0 for o in out)


def test_config0_full(ctx, oracle):
    rays, pix = synth.config0(seed=0)
    ref = oracle_run(oracle, rays, pix)
    out64, _ = run(ctx, rays, pix, "f64")
    assert cases.rel_l2(out64, ref) < F64_TOL
    out32, st = run(ctx, rays, pix, "f32pr")
    assert st["path"] == xrt_rs.XK_PATH_F32PR
    assert cases.rel_l2(out32, ref) < PR_TOL
    assert cases.rel_l2_intensity(out32, ref) < PR_TOL


def test_deterministic(ctx):
    rays, pix = synth.config0(seed=1)
    a, _ = run(ctx, rays, pix, "f32pr")
    b, _ = run(ctx, rays, pix, "f32pr")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    a, _ = run(ctx, rays, pix, "f64")
    b, _ = run(ctx, rays, pix, "f64")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_config1_subsample_f64_vs_oracle(ctx, oracle):
    """2^20 rays; 128 seeded screen points of the 512x512 grid."""
    rays, screen = synth.config1(seed=0)
    sub, _ = synth.subsample_screen(screen, 128, seed=5)
    ref = oracle_run(oracle, rays, sub)
    out64, _ = run(ctx, rays, sub, "f64")
    assert cases.rel_l2(out64, ref) < F64_TOL


def test_config1_full_f32pr_vs_f64(ctx):
    """Full 512x512 field: F32PR against the GPU F64 path (itself pinned to the
    oracle by the subsample test above)."""
    rays, screen = synth.config1(seed=0)
    ref, st64 = run(ctx, rays, screen, "f64")
    out, st = run(ctx, rays, screen, "f32pr")
    assert st["path"] == xrt_rs.XK_PATH_F32PR
    err = cases.rel_l2(out, ref)
    err_i = cases.rel_l2_intensity(out, ref)
    print(f"config1 rel_l2 field={err:.3e} intensity={err_i:.3e} "
          f"f64 {st64['gpu_ms']:.1f} ms, f32pr {st['gpu_ms']:.1f} ms, stats={st}")
    assert err < PR_TOL
    assert err_i < PR_TOL


def test_kirchhoff_gpu_records(ctx, oracle, golden_case):
    """gpu::kirchhoff::kirchhoff_gpu on the fixture (golden_gpu_kirchhoff.rs:103-182)."""
    r = golden_case["rays"]
    recs = np.zeros(5, dtype=xrt_rs.GPU_RAY_DTYPE)
    for k in xrt_rs.GPU_RAY_DTYPE.names:
        recs[k] = r[k]
    pix = np.zeros(3, dtype=xrt_rs.GPU_PIXEL_DTYPE)
    for k in "xyz":
        pix[k] = golden_case["pixels"][k]
    es, ep = xrt_rs.kirchhoff_gpu(ctx, recs, pix)
    es2, ep2 = xrt_rs.kirchhoff_auto(recs, pix)
    f32 = [recs[k].astype(np.float64) for k in cases.RAY_FIELDS]
    ref = oracle.plain_f64(f32, [pix[k].astype(np.float64) for k in "xyz"])
    for i in range(3):
        c = ref[0][i] + 1j * ref[1][i]
        assert abs(es[i]) > 1e-10
        assert abs(es[i] - c) / abs(c) < 1e-4
        assert abs(es2[i] - c) / abs(c) < 1e-4


@pytest.mark.parametrize("n_rays,n_pix", [(0, 7), (1, 1), (3001, 257), (40_000, 4099)])
def test_kirchhoff_gpu_records_match_columns(ctx, n_rays, n_pix):
    """The record entry point widens on the device and interleaves the field
    there: identical, bit for bit, to the column entry point on the same
    (f32-rounded) values; no rays gives a zero field."""
    rays, pix = synth.config0(seed=3)
    rng = np.random.default_rng(n_rays + n_pix)
    ri = rng.integers(0, len(rays["x"]), n_rays)
    pi = rng.integers(0, len(pix["x"]), n_pix)
    recs = np.zeros(n_rays, dtype=xrt_rs.GPU_RAY_DTYPE)
    for k in xrt_rs.GPU_RAY_DTYPE.names:
        recs[k] = rays[k][ri]
    px = np.zeros(n_pix, dtype=xrt_rs.GPU_PIXEL_DTYPE)
    for k in "xyz":
        px[k] = pix[k][pi]
    es, ep = xrt_rs.kirchhoff_gpu(ctx, recs, px)
    wide_r = {k: recs[k].astype(np.float64) for k in cases.RAY_FIELDS}
    wide_p = {k: px[k].astype(np.float64) for k in "xyz"}
    out, _ = run(ctx, wide_r, wide_p, "f32pr")
    assert np.array_equal(es.real, out[0]) and np.array_equal(es.imag, out[1])
    assert np.array_equal(ep.real, out[2]) and np.array_equal(ep.imag, out[3])
    if n_rays == 0:
        assert not np.any(es) and not np.any(ep)


@pytest.fixture
def sweep_ctx(ctx):
    yield ctx
    ctx.set_option("sweep", -1)


@pytest.mark.parametrize("sweep", [0, 1, 2])
def test_both_sweeps_config0(sweep_ctx, oracle, sweep):
    """The SFU-reciprocal sweep and the packed f32x2 sweeps (quadratic and
    linear series reciprocal)."""
    sweep_ctx.set_option("sweep", sweep)
    rays, pix = synth.config0(seed=3)
    ref = oracle_run(oracle, rays, pix)
    out, st = run(sweep_ctx, rays, pix, "f32pr")
    assert st["sweep"] == sweep
    assert cases.rel_l2(out, ref) < PR_TOL
    assert cases.rel_l2_intensity(out, ref) < PR_TOL


@pytest.mark.parametrize("sweep", [0, 1, 2])
def test_both_sweeps_general_normals(sweep_ctx, oracle, sweep):
    sweep_ctx.set_option("sweep", sweep)
    rays, pix = cases.random_case(2000, 300, seed=21, general_normals=True)
    out, st = run(sweep_ctx, rays, pix, "f32pr")
    assert st["sweep"] == sweep
    assert cases.rel_l2(out, oracle_run(oracle, rays, pix)) < PR_TOL


def test_phase_budget_option(sweep_ctx, oracle):
    """A tighter residual-phase budget gives finer ray chunks and the same field."""
    rays, pix = synth.config0(seed=4)
    ref = oracle_run(oracle, rays, pix)
    sweep_ctx.set_option("phase_budget", 32.0)
    try:
        out, st = run(sweep_ctx, rays, pix, "f32pr")
    finally:
        sweep_ctx.set_option("phase_budget", 512.0)
    assert st["phase_bound_rad"] <= 32.0 + 1e-9
    assert cases.rel_l2(out, ref) < PR_TOL


@pytest.mark.parametrize("energy,dist", [(30000.0, 20000.0), (30000.0, 100.0), (1000.0, 20000.0)])
def test_f32pr_extreme_cells_vs_extended_oracle(ctx, oracle, energy, dist):
    """Corners of the E <= 30 keV, d <= 20 m range, 4096 rays x 32x32 screen.
    The FP32 phase-reduced form is compared with the extended-precision oracle;
    the FP64 formula's own distance from it is printed beside."""
    rays, screen, meta = synth.config2_cell(energy, dist, seed=17, n_rays=4096, grid=32)
    rl, pl = cases.as_lists(rays, screen)
    exact = oracle.kahan_ld(rl, pl)
    out, st = run(ctx, rays, screen, "f32pr")
    err = cases.rel_l2(out, exact)
    f64_err = cases.rel_l2(oracle.kahan_f64(rl, pl), exact)
    print(f"E={energy} d={dist}: f32pr vs exact {err:.2e}, fp64 formula vs exact {f64_err:.2e}, "
          f"chunks={st['n_chunks']} path={st['path']}")
    assert err < PR_TOL


def test_autotune_keeps_results_and_restores_options(ctx, oracle):
    torch = pytest.importorskip("torch")
    rays, pix = synth.config0(seed=6)
    rl, pl = cases.as_lists(rays, pix)
    d_r = [torch.from_numpy(a).cuda() for a in rl]
    d_p = [torch.from_numpy(a).cuda() for a in pl]
    d_o = [torch.zeros(len(pl[0]), dtype=torch.float64, device="cuda") for _ in range(4)]
    res = xrt_rs.autotune(d_r, d_p, d_o, ctx=ctx, budget_ms=50.0, apply=False)
    assert res["trials"] >= 1 and res["best_ms"] <= res["default_ms"] + 1e-9
    assert res["phase_budget"] <= 512.0
    out = [t.cpu().numpy() for t in d_o]
    assert cases.rel_l2(out, oracle.kahan_ld(rl, pl)) < PR_TOL
    # apply=False left the context's defaults in force
    _, st = run(ctx, rays, pix, "f32pr")
    assert st["phase_bound_rad"] <= 512.0 + 1e-9


def test_f64_reduction_option_keeps_parity(ctx, oracle):
    """The FMA-based reduction of the FP64 phase (option "f64_reduction")
    gives the same 1e-10 parity as the library sin/cos, at 1 m and at the far
    end of the range (25 keV, 8 m)."""
    rays, pix = synth.config0(seed=2)
    far, fpix, _ = synth.config3(seed=0, count=2, ray_range=(300, 30000), pix_range=(17, 4000))[1]
    ctx.set_option("f64_reduction", 1)
    try:
        for r, p in ((rays, pix), (far, fpix)):
            out, st = run(ctx, r, p, "f64")
            assert st["path"] == xrt_rs.XK_PATH_F64
            assert cases.rel_l2(out, oracle_run(oracle, r, p)) < F64_TOL
    finally:
        ctx.set_option("f64_reduction", 0)


def test_linear_series_chosen_only_where_its_error_is_negligible(sweep_ctx, oracle):
    """Automatic sweep: the linear series where |e|^2 x budget stays below a
    tenth of the tolerance (e = u.rho / |q| <= b / (d - b), b the ray-chunk
    radius), as on the 10 keV, 1 m workload; the quadratic one where chunks
    are large for their distance (1 keV, 100 mm, a screen a few microns wide,
    so e ~ 1e-3). Both within the tolerance of the extended-precision oracle."""
    far, far_pix = synth.config1(seed=2, n_rays=1 << 14, grid=32)
    near = synth.gaussian_aperture(1 << 14, 0.1, 1000.0, 30000.0, seed=3)
    near_pix = synth.line_screen(64, 0.002, 100.0)
    for rays, pix, want in ((far, far_pix, 2), (near, near_pix, 1)):
        out, st = run(sweep_ctx, rays, pix, "f32pr")
        assert st["sweep"] == want, st
        rl, pl = cases.as_lists(rays, pix)
        assert cases.rel_l2(out, oracle.kahan_ld(rl, pl)) < PR_TOL


def test_autotune_cache_per_bucket(oracle):
    """xk_autotune with apply keeps its best settings for the problem's bucket
    (energy, distance, ray count, screen count): later solves of that bucket,
    single or batched, report `tuned` and stay within the tolerance of the
    extended-precision oracle; a solve of another bucket, or with the cache
    switched off, runs the defaults bit for bit as before."""
    torch = pytest.importorskip("torch")
    ctx = xrt_rs.GpuContext.new(0)
    try:
        rays, pix = synth.config0(seed=7)
        rl, pl = cases.as_lists(rays, pix)
        default, st0 = run(ctx, rays, pix, "f32pr")
        assert st0["tuned"] == 0
        d_r = [torch.from_numpy(a).cuda() for a in rl]
        d_p = [torch.from_numpy(a).cuda() for a in pl]
        d_o = [torch.zeros(len(pl[0]), dtype=torch.float64, device="cuda") for _ in range(4)]
        res = xrt_rs.autotune(d_r, d_p, d_o, ctx=ctx, budget_ms=200.0, apply=True)
        assert res["trials"] >= 1
        out, st = run(ctx, rays, pix, "f32pr")
        assert st["tuned"] == 1, (st, res)
        exact = oracle.kahan_ld(rl, pl)
        assert cases.rel_l2(out, exact) < PR_TOL
        assert cases.rel_l2_intensity(out, exact) < PR_TOL
        # The same bucket in a batch.
        b = xrt_rs.Batch([(rays, pix)], path="f32pr", ctx=ctx)
        outs = b.run()
        assert b.plan(0)["tuned"] == 1
        assert all(np.array_equal(x, y) for x, y in zip(outs[0], out))
        b.close()
        # Another bucket (100x the screen distance) is not tuned.
        far = dict(pix, z=pix["z"] * 100.0)
        _, st_far = run(ctx, rays, far, "f32pr")
        assert st_far["tuned"] == 0
        # Cache off: the defaults, bit for bit.
        ctx.set_option("use_tuned", 0)
        again, st2 = run(ctx, rays, pix, "f32pr")
        assert st2["tuned"] == 0
        assert all(np.array_equal(x, y) for x, y in zip(again, default))
        ctx.set_option("use_tuned", 1)
        ctx.set_option("clear_tuned", 1)
        _, st3 = run(ctx, rays, pix, "f32pr")
        assert st3["tuned"] == 0
    finally:
        ctx.close()
