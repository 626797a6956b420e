"""FP32 phase-reduced path at its worst cases, against the extended-precision oracle.

The FP32 residual phase of a pair is bounded by the planner's phase budget
(512 rad by default); its rounding and the SFU sine/cosine of it are where the
FP32 form loses accuracy. On noise-like fields these per-pair errors average
out over many rays. On coherent fields they do not: a few rays in phase, a
point source (spherical wave) and a focus (every ray in phase at one screen
point) put the whole error of a handful of pairs into the result. These tests
run those fields at the corners of the E <= 30 keV, d <= 20 m range, and every
cell of the energy x distance sweep, and assert rel L2 <= 1e-4 on the complex
field and on |E|^2 against ``oracle.kahan_ld`` (the reference formula,
src/waves/diffraction.rs:67-117, with the phase in extended precision). Each
test prints its margin (1e-4 / error).
"""
import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import synth

pytestmark = pytest.mark.gpu

PR_TOL = 1e-4
CORNERS = [(1000.0, 100.0), (1000.0, 20000.0), (30000.0, 100.0), (30000.0, 20000.0)]


def _k(energy):
    return synth.wavenumber(energy)


def _screen(dist, half, n=193):
    """A line of n points across the axis and a 9 x 9 patch around it."""
    x = np.linspace(-half, half, n)
    g = np.linspace(-half / 4, half / 4, 9)
    gx, gy = np.repeat(g, 9), np.tile(g, 9)
    return cases.pixels_from(np.concatenate([x, gx]), np.concatenate([np.zeros(n), gy]),
                             np.full(n + 81, dist))


def _half_width(energy, dist):
    """Screen half-width: a few diffraction widths of a 0.1 mm aperture,
    between 0.05 mm and 2 mm."""
    lam = 2 * np.pi / _k(energy)
    return float(np.clip(8 * lam * dist / 0.1, 0.05, 2.0))


def _phase_ld(energy, d):
    """k * d reduced to [0, 2 pi) in extended precision (d in mm, any shape)."""
    k = np.longdouble(energy) / np.longdouble("1973.2697177417986") * np.longdouble(1e7)
    ph = k * np.asarray(d, dtype=np.longdouble)
    two_pi = 2 * np.longdouble("3.14159265358979323846264338327950288")
    return np.asarray(np.mod(ph, two_pi), dtype=np.float64)


def coherent_line(n, width, energy):
    """n rays on the x axis across `width` mm, all with es = 1, ep = 0.1."""
    x = np.linspace(-width / 2, width / 2, n) if n > 1 else np.zeros(1)
    return cases.rays_from(x, es=1.0 + 0j, ep=0.1 + 0j, energy=energy)


def point_source(n, energy, radius, seed=3):
    """n rays on a 0.2 mm disk lit by a point source `radius` mm behind it:
    es = exp(i k |r - s|), a diverging spherical wave."""
    rng = np.random.default_rng(seed)
    rad = 0.1 * np.sqrt(rng.uniform(0, 1, n))
    ang = rng.uniform(0, 2 * np.pi, n)
    x, y = rad * np.cos(ang), rad * np.sin(ang)
    d = np.sqrt(x.astype(np.longdouble) ** 2 + y.astype(np.longdouble) ** 2
                + np.longdouble(radius) ** 2)
    es = np.exp(1j * _phase_ld(energy, d))
    return cases.rays_from(x, y, es=es, ep=0.1 * es, energy=energy)


def focus(n, energy, dist, seed=4):
    """n rays on a 0.2 mm disk with es = exp(-i k |f - r|), f = (0, 0, dist):
    every ray arrives in phase at the screen centre."""
    rng = np.random.default_rng(seed)
    rad = 0.1 * np.sqrt(rng.uniform(0, 1, n))
    ang = rng.uniform(0, 2 * np.pi, n)
    x, y = rad * np.cos(ang), rad * np.sin(ang)
    d = np.sqrt(x.astype(np.longdouble) ** 2 + y.astype(np.longdouble) ** 2
                + np.longdouble(dist) ** 2)
    es = np.exp(-1j * _phase_ld(energy, d))
    return cases.rays_from(x, y, es=es, ep=0.1 * es, energy=energy)


def _check(ctx, oracle, rays, pix, label):
    rl, pl = cases.as_lists(rays, pix)
    exact = oracle.kahan_ld(rl, pl)
    out, st = xrt_rs.diffraction_integral(rl, pl, path="f32pr", ctx=ctx, return_stats=True)
    assert st["path"] == xrt_rs.XK_PATH_F32PR, (label, st)
    err = cases.rel_l2(out, exact)
    err_i = cases.rel_l2_intensity(out, exact)
    worst = max(err, err_i)
    print(f"{label}: field {err:.2e} |E|^2 {err_i:.2e} margin {PR_TOL / max(worst, 1e-30):.1f}x "
          f"chunks={st['n_chunks']} phase_bound={st['phase_bound_rad']:.1f}")
    assert err <= PR_TOL, label
    assert err_i <= PR_TOL, label
    return worst


@pytest.mark.parametrize("energy,dist", CORNERS)
@pytest.mark.parametrize("n", [1, 2, 10, 100])
@pytest.mark.parametrize("width", [0.01, 0.2, 2.0])
def test_coherent_rays_on_axis(ctx, oracle, energy, dist, n, width):
    if n == 1 and width != 0.01:
        pytest.skip("one ray has no width")
    rays = coherent_line(n, width, energy)
    pix = _screen(dist, _half_width(energy, dist))
    _check(ctx, oracle, rays, pix, f"{n} rays over {width} mm, E={energy} d={dist}")


@pytest.mark.parametrize("energy,dist", CORNERS)
def test_point_source(ctx, oracle, energy, dist):
    rays = point_source(1000, energy, radius=1000.0)
    pix = _screen(dist, _half_width(energy, dist))
    _check(ctx, oracle, rays, pix, f"point source, E={energy} d={dist}")


@pytest.mark.parametrize("energy,dist", CORNERS)
def test_focus(ctx, oracle, energy, dist):
    rays = focus(1000, energy, dist)
    pix = _screen(dist, _half_width(energy, dist) / 4)
    _check(ctx, oracle, rays, pix, f"focus, E={energy} d={dist}")


@pytest.mark.parametrize("energy", synth.CONFIG2_ENERGIES)
@pytest.mark.parametrize("dist", synth.CONFIG2_DISTANCES)
def test_config2_every_cell(ctx, oracle, energy, dist):
    """Every cell of the energy x distance sweep: 2^16 rays x a 64 x 64 grid of
    +-1 mm (Gaussian aperture sigma ~ U(0.02, 0.2) mm, spherical phase of radius
    R ~ U(10, 50) m), checked on 256 seeded screen points."""
    seed = int(energy) // 1000 * 100 + int(dist) // 100
    rays, screen, meta = synth.config2_cell(energy, dist, seed=seed, n_rays=1 << 16, grid=64)
    rl, pl = cases.as_lists(rays, screen)
    out, st = xrt_rs.diffraction_integral(rl, pl, path="f32pr", ctx=ctx, return_stats=True)
    assert st["path"] == xrt_rs.XK_PATH_F32PR
    sub, idx = synth.subsample_screen(screen, 256, seed=seed + 1)
    exact = oracle.kahan_ld(rl, [sub[k] for k in cases.PIXEL_FIELDS])
    got = [o[idx] for o in out]
    err = cases.rel_l2(got, exact)
    err_i = cases.rel_l2_intensity(got, exact)
    print(f"cell E={energy} d={dist} sigma={meta['sigma_mm']:.3f}: field {err:.2e} "
          f"|E|^2 {err_i:.2e} margin {PR_TOL / max(err, err_i, 1e-30):.1f}x "
          f"chunks={st['n_chunks']}")
    assert err <= PR_TOL
    assert err_i <= PR_TOL
