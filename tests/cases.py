"""Parity inputs restated from the reference's own tests and bench.

Each builder returns (rays, pixels) as dicts of float64 arrays in the
RAY_FIELDS / PIXEL_FIELDS layout and cites the reference test it follows.
"""
import numpy as np

RAY_FIELDS = ("x", "y", "z", "nx", "ny", "nz", "nl", "es_re", "es_im", "ep_re", "ep_im", "energy")
PIXEL_FIELDS = ("x", "y", "z")


def rays_from(x, y=None, z=None, n=(0.0, 0.0, 1.0), nl=1.0, es=1.0 + 0j, ep=0j, energy=10000.0):
    x = np.asarray(x, dtype=np.float64)
    k = len(x)

    def full(v):
        a = np.asarray(v)
        return np.broadcast_to(a, (k,)).astype(a.dtype if a.dtype.kind == "c" else np.float64).copy()

    es = np.broadcast_to(np.asarray(es, dtype=np.complex128), (k,))
    ep = np.broadcast_to(np.asarray(ep, dtype=np.complex128), (k,))
    return {
        "x": x.copy(),
        "y": full(0.0 if y is None else y).astype(np.float64),
        "z": full(0.0 if z is None else z).astype(np.float64),
        "nx": np.full(k, n[0]), "ny": np.full(k, n[1]), "nz": np.full(k, n[2]),
        "nl": full(nl).astype(np.float64),
        "es_re": es.real.copy(), "es_im": es.imag.copy(),
        "ep_re": ep.real.copy(), "ep_im": ep.imag.copy(),
        "energy": full(energy).astype(np.float64),
    }


def pixels_from(x, y, z):
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    k = len(x)
    return {"x": x, "y": np.broadcast_to(np.asarray(y, dtype=np.float64), (k,)).copy(),
            "z": np.broadcast_to(np.asarray(z, dtype=np.float64), (k,)).copy()}


def single_ray_single_pixel():
    """src/waves/diffraction.rs:123-149."""
    return rays_from([0.0]), pixels_from([0.0], 1000.0, 0.0)


def parallel_pixels():
    """src/waves/diffraction.rs:151-194."""
    i = np.arange(100)
    j = np.arange(50)
    return rays_from((i - 50.0) * 0.01), pixels_from((j - 25.0) * 0.02, 1000.0, 0.0)


def ray_at_pixel():
    """src/waves/diffraction.rs:196-225: path = 0 is skipped."""
    return (rays_from([1.0], [2.0], [3.0], es=1 + 0j, ep=1 + 0j), pixels_from([1.0], 2.0, 3.0))


def kahan_stability(n=10_000):
    """src/waves/diffraction.rs:227-285."""
    i = np.arange(n)
    return rays_from((i - n / 2.0) * 0.001, es=(1.0 / n) + 0j), pixels_from([0.0], 0.0, 100.0)


def large_ray_count(n=50_000):
    """src/waves/diffraction.rs:307-351."""
    i = np.arange(n)
    return (rays_from((i - n / 2.0) * 0.0001, es=(1.0 / n) + 0j),
            pixels_from([0.0, 0.1], 0.0, 100.0))


def polychromatic():
    """src/waves/diffraction.rs:353-397."""
    return (rays_from([0.0, 0.01], energy=np.array([8000.0, 12000.0])),
            pixels_from([0.0], 0.0, 100.0))


def symmetry():
    """tests/golden_diffraction.rs:79-116."""
    return rays_from([0.0], es=1 + 0j, ep=1 + 0j), pixels_from([-0.01, 0.01], 0.0, 1000.0)


def gpu_short_distance():
    """tests/golden_gpu_kirchhoff.rs:184-247 (f32 GpuRay values)."""
    r = rays_from([0.0, 0.01], energy=1000.0, es=np.array([1.0 + 0j, 0.8 - 0.1j]),
                  ep=np.array([0.5 + 0.1j, 0.6 + 0j]))
    return r, pixels_from([0.0, 0.005], 0.0, 0.1)


def gpu_extreme_distance():
    """tests/golden_gpu_kirchhoff.rs:329-391: one pixel at 10 m."""
    r = rays_from([0.0, 0.01], es=np.array([1.0 + 0j, 0.8 + 0.1j]),
                  ep=np.array([0.5 + 0j, 0.6 - 0.1j]))
    return r, pixels_from([0.0], 0.0, 10000.0)


def bench_case(n_rays, n_pix):
    """benches/diffraction.rs:6-37: rays on a line at 0.01 mm pitch, pixels at
    0.02 mm pitch on the line y = 1000."""
    i = np.arange(n_rays)
    j = np.arange(n_pix)
    return (rays_from((i - n_rays / 2.0) * 0.01),
            pixels_from((j - n_pix / 2.0) * 0.02, 1000.0, 0.0))


BENCH_SIZES = ((100, 50), (500, 100), (1000, 200), (5000, 100))


def random_case(n_rays, n_pix, seed, dist=1000.0, energy=10000.0, spread=0.05, general_normals=False):
    """Seeded random rays and screen points (odd sizes hit every tile edge)."""
    rng = np.random.default_rng(seed)
    x = rng.normal(0, spread, n_rays)
    y = rng.normal(0, spread, n_rays)
    z = rng.normal(0, spread * 0.1, n_rays) if general_normals else np.zeros(n_rays)
    es = rng.uniform(0.5, 1.0, n_rays) + 1j * rng.uniform(-0.1, 0.1, n_rays)
    ep = rng.uniform(0.5, 1.0, n_rays) + 1j * rng.uniform(-0.1, 0.1, n_rays)
    r = rays_from(x, y, z, es=es, ep=ep, energy=energy)
    if general_normals:
        nrm = rng.normal(0, 0.05, (n_rays, 3))
        nrm[:, 2] += 1.0
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        r["nx"], r["ny"], r["nz"] = nrm[:, 0].copy(), nrm[:, 1].copy(), nrm[:, 2].copy()
        r["nl"] = nrm[:, 2].copy()
    px = rng.uniform(-0.3, 0.3, n_pix)
    py = rng.uniform(-0.3, 0.3, n_pix)
    return r, pixels_from(px, py, np.full(n_pix, dist))


def as_lists(rays, pixels):
    return [rays[k] for k in RAY_FIELDS], [pixels[k] for k in PIXEL_FIELDS]


def field_c(out):
    """(es_re, es_im, ep_re, ep_im) -> complex (es, ep)."""
    return np.asarray(out[0]) + 1j * np.asarray(out[1]), np.asarray(out[2]) + 1j * np.asarray(out[3])


def rel_l2(out, ref):
    """Relative L2 error over the complex field (Es and Ep together)."""
    a = np.concatenate(field_c(out))
    b = np.concatenate(field_c(ref))
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def rel_l2_intensity(out, ref):
    """Relative L2 error of |Es|^2 + |Ep|^2."""
    ea, pa = field_c(out)
    eb, pb = field_c(ref)
    ia = np.abs(ea) ** 2 + np.abs(pa) ** 2
    ib = np.abs(eb) ** 2 + np.abs(pb) ** 2
    den = np.linalg.norm(ib)
    return float(np.linalg.norm(ia - ib) / den) if den > 0 else float(np.linalg.norm(ia - ib))


def beam_case(n, seed, amplitudes=True, dist_y=2000.0):
    """A seeded beam after a mirror, in the column layout beam_to_diffraction_rays
    reads (x, y, z, a, b, c, e, es/ep), with per-ray normals and a `good`
    subset in shuffled order with repeats — the shape of
    tests/pipeline.rs:13-54 (source -> flat mirror -> screen at y = 2000)."""
    rng = np.random.default_rng(seed)
    d = rng.normal(0, 1e-4, (n, 3))
    d[:, 1] += 1.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    beam = {"x": rng.normal(0, 0.1, n), "y": rng.normal(0, 1e-3, n), "z": rng.normal(0, 0.1, n),
            "a": d[:, 0].copy(), "b": d[:, 1].copy(), "c": d[:, 2].copy(),
            "e": np.full(n, 10000.0)}
    if amplitudes:
        es = rng.uniform(0.5, 1.0, n) * np.exp(1j * rng.uniform(-0.3, 0.3, n))
        ep = 0.1 * es
        beam.update(es_re=es.real.copy(), es_im=es.imag.copy(), ep_re=ep.real.copy(),
                    ep_im=ep.imag.copy())
    nrm = rng.normal(0, 0.02, (n, 3))
    nrm[:, 1] += 1.0
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    good = rng.permutation(n)[: max(1, (9 * n) // 10)]
    good = np.concatenate([good, good[:3]])  # repeats are allowed
    return beam, nrm, good.astype(np.uint64)
