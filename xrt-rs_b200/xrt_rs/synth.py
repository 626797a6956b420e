"""Seeded synthetic Kirchhoff workloads.

The reference has no dataset for this path; these generators build the
apertures and screens of the benchmark configurations from their stated
shapes, sizes and distributions:

* Gaussian aperture: rays on the plane z = 0, x, y ~ N(0, sigma), normal
  (0, 0, 1), direction +z (so nl = 1), Es = exp(-(x^2+y^2)/(4 sigma^2)) *
  exp(i k (x^2+y^2) / (2 R)), Ep = 0.1 Es, one energy per solve.
* Screens on the plane z = d: a 1-D line along x, or a square grid in row-major
  order with x outer and y inner (the ordering of prepare_wave,
  src/waves/prepare_wave.rs:40-68).

Every array is float64; rays come back as a dict keyed by RAY_FIELDS and
screens as a dict keyed by PIXEL_FIELDS.
"""
from __future__ import annotations

import math

import numpy as np

CHBAR = 1973.2697177417986  # eV*Angstrom, src/core/consts.rs:74


def wavenumber(energy_ev: float) -> float:
    """k = E / CHBAR * 1e7 in 1/mm, rounded as the reference rounds it."""
    return energy_ev / CHBAR * 1e7


def gaussian_aperture(n: int, sigma_mm: float, energy_ev: float, radius_mm: float, seed: int):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, sigma_mm, n)
    y = rng.normal(0.0, sigma_mm, n)
    k = wavenumber(energy_ev)
    r2 = x * x + y * y
    mag = np.exp(-r2 / (4.0 * sigma_mm * sigma_mm))
    ph = k * r2 / (2.0 * radius_mm)
    es = mag * np.exp(1j * ph)
    ep = 0.1 * es
    zeros = np.zeros(n)
    ones = np.ones(n)
    return {
        "x": x, "y": y, "z": zeros.copy(),
        "nx": zeros.copy(), "ny": zeros.copy(), "nz": ones.copy(),
        "nl": ones.copy(),
        "es_re": es.real.copy(), "es_im": es.imag.copy(),
        "ep_re": ep.real.copy(), "ep_im": ep.imag.copy(),
        "energy": np.full(n, float(energy_ev)),
    }


def line_screen(n: int, half_mm: float, z_mm: float):
    x = np.linspace(-half_mm, half_mm, n)
    return {"x": x, "y": np.zeros(n), "z": np.full(n, float(z_mm))}


def grid_screen(nx: int, ny: int, half_mm: float, z_mm: float):
    gx = np.linspace(-half_mm, half_mm, nx)
    gy = np.linspace(-half_mm, half_mm, ny)
    x = np.repeat(gx, ny)
    y = np.tile(gy, nx)
    return {"x": x, "y": y, "z": np.full(nx * ny, float(z_mm))}


def subsample_screen(screen, count: int, seed: int):
    """A seeded subset of screen points (for CPU-oracle checks of big screens)."""
    m = len(screen["x"])
    if count >= m:
        return screen, np.arange(m)
    idx = np.sort(np.random.default_rng(seed).choice(m, size=count, replace=False))
    return {k: np.ascontiguousarray(v[idx]) for k, v in screen.items()}, idx


# ---- the benchmark configurations -------------------------------------------

def config0(seed: int = 0):
    """10,000 rays, sigma 0.05 mm, R = 30 m, 10 keV; 256-point line +-0.5 mm at 1 m."""
    rays = gaussian_aperture(10_000, 0.05, 10_000.0, 30_000.0, seed)
    return rays, line_screen(256, 0.5, 1000.0)


def config1(seed: int = 0, n_rays: int = 1 << 20, grid: int = 512):
    """2^20 rays, sigma 0.1 mm, R = 30 m, 10 keV; 512x512 grid +-0.5 mm at 1 m."""
    rays = gaussian_aperture(n_rays, 0.1, 10_000.0, 30_000.0, seed)
    return rays, grid_screen(grid, grid, 0.5, 1000.0)


CONFIG2_ENERGIES = (1_000.0, 5_000.0, 10_000.0, 20_000.0, 30_000.0)
CONFIG2_DISTANCES = (100.0, 1_000.0, 5_000.0, 20_000.0)


def config2_cell(energy_ev: float, dist_mm: float, seed: int, n_rays: int = 1 << 18,
                 grid: int = 256):
    """One precision-sweep cell: sigma ~ U(0.02, 0.2) mm, R ~ U(10, 50) m."""
    rng = np.random.default_rng(seed)
    sigma = float(rng.uniform(0.02, 0.2))
    radius = float(rng.uniform(10_000.0, 50_000.0))
    rays = gaussian_aperture(n_rays, sigma, energy_ev, radius, seed + 1)
    meta = {"energy_ev": energy_ev, "dist_mm": dist_mm, "sigma_mm": sigma, "radius_mm": radius}
    return rays, grid_screen(grid, grid, 1.0, dist_mm), meta


def _log_uniform(rng, lo, hi):
    return float(math.exp(rng.uniform(math.log(lo), math.log(hi))))


def config3(seed: int = 0, count: int = 64, ray_range=(1e3, 1e6), pix_range=(64, 262144)):
    """Uneven batch: log-uniform ray and screen counts, square or 1-D grids."""
    rng = np.random.default_rng(seed)
    solves = []
    for i in range(count):
        n = int(round(_log_uniform(rng, *ray_range)))
        m = int(round(_log_uniform(rng, *pix_range)))
        energy = float(rng.uniform(5_000.0, 25_000.0))
        dist = float(rng.uniform(500.0, 10_000.0))
        sigma = float(rng.uniform(0.02, 0.2))
        radius = float(rng.uniform(10_000.0, 50_000.0))
        square = bool(rng.integers(0, 2))
        rays = gaussian_aperture(n, sigma, energy, radius, seed * 1000 + i)
        if square:
            side = max(1, int(round(math.sqrt(m))))
            screen = grid_screen(side, side, 1.0, dist)
        else:
            screen = line_screen(m, 1.0, dist)
        solves.append((rays, screen, {"energy_ev": energy, "dist_mm": dist, "sigma_mm": sigma,
                                      "radius_mm": radius, "square": square}))
    return solves


def config4_requests(seed: int = 0, rate_hz: float = 200.0, duration_s: float = 60.0,
                     ray_range=(1e4, 2e6), pix_range=(256, 1e6), reuse: float = 0.3):
    """Poisson request stream (arrival time, sizes, energy, distance, reuse flag).

    Returns descriptors only; ``materialize`` builds the arrays of one request.
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    while True:
        t += float(rng.exponential(1.0 / rate_hz))
        if t >= duration_s:
            break
        reuse_set = bool(reqs) and rng.uniform() < reuse
        n = int(round(_log_uniform(rng, *ray_range)))
        m = int(round(_log_uniform(rng, *pix_range)))
        reqs.append({
            "t": t,
            "n_rays": n,
            "n_pix": m,
            "energy_ev": float(rng.uniform(1_000.0, 30_000.0)),
            "dist_mm": float(rng.uniform(100.0, 20_000.0)),
            "sigma_mm": float(rng.uniform(0.02, 0.2)),
            "radius_mm": float(rng.uniform(10_000.0, 50_000.0)),
            "reuse_of": int(rng.integers(0, len(reqs))) if reuse_set else -1,
            "seed": int(rng.integers(0, 2**31 - 1)),
        })
    return reqs
