"""The Fresnel oracle (a restatement of src/waves/fresnel.rs:53-106) against
closed-form fields: one and two point sources, and a row of equal rays at the
Talbot pitch, whose sum is a geometric series evaluated in closed form
(tests/fresnel_closed.py). The bar is 1e-12 relative L2, widened only by the
FP64 rounding of the largest phase the sum forms (8 * 2^-53 * phase), which
the reference's own arithmetic carries."""
import numpy as np
import pytest

import fresnel_closed as F

EPS = 2.0 ** -53

# (energy eV, distance mm, screen (x_min, x_max, nx, z_min, z_max, nz))
GEOMS = [
    (10000.0, 1000.0, (-0.3, 0.25, 41, -0.2, 0.2, 23)),
    (1000.0, 20000.0, (-1.0, 1.0, 64, -0.5, 0.5, 17)),
    (8000.0, 5000.0, (-0.4, 0.4, 33, 0.0, 0.0, 1)),
    (30000.0, 100.0, (-0.05, 0.05, 29, -0.04, 0.04, 31)),
]


def max_phase(energy, dist, x, z, sc):
    xp, zp = F.screen_coords(*sc)
    dx = max(abs(xp.max() - np.min(x)), abs(xp.min() - np.max(x)))
    dz = max(abs(zp.max() - np.min(z)), abs(zp.min() - np.max(z)))
    return float(F.a_coef(energy, dist)) * (dx * dx + dz * dz)


def tol(base, energy, dist, x, z, sc):
    return max(base, 8 * EPS * max_phase(energy, dist, x, z, sc))


def sources(kind, energy, dist):
    """(x, z, es, exact field function) of a closed-form case."""
    if kind == "one":
        x, z, e = np.array([0.013]), np.array([-0.021]), np.array([0.7 - 0.2j])
    elif kind == "two":
        x, z, e = (np.array([0.013, -0.05]), np.array([-0.021, 0.03]),
                   np.array([0.7 - 0.2j, -0.1 + 0.4j]))
    else:
        n = 16 if kind == "row16" else 97
        x, z, e, f = F.talbot_row(n, -0.11 * F.talbot_pitch(energy, dist) / 0.0158, 0.02,
                                  0.9 + 0.1j, energy, dist)
        return x, z, e, f
    return x, z, e, (lambda xp, zp: F.point_sources(x, z, e, energy, dist, xp, zp))


def oracle_field(oracle, x, z, e, energy, dist, sc):
    re, im = oracle.fresnel(x, z, e.real, e.imag, energy, dist, *sc)
    return re + 1j * im


@pytest.mark.parametrize("geom", range(len(GEOMS)))
@pytest.mark.parametrize("kind", ["one", "two", "row16", "row97"])
def test_oracle_matches_closed_form(oracle, geom, kind):
    energy, dist, sc = GEOMS[geom]
    x, z, e, exact = sources(kind, energy, dist)
    xp, zp = F.screen_coords(*sc)
    got = oracle_field(oracle, x, z, e, energy, dist, sc)
    err = F.rel_l2(got, exact(xp, zp))
    bar = tol(1e-12, energy, dist, x, z, sc)
    assert err <= bar, (err, bar)


def test_talbot_row_closed_form_is_the_series():
    """The geometric-series closed form equals the direct sum of its terms."""
    energy, dist = 10000.0, 1000.0
    x, z, e, exact = F.talbot_row(12, 0.003, -0.01, 1.0 + 0.0j, energy, dist)
    xp = np.linspace(-0.2, 0.2, 17)
    zp = np.linspace(-0.1, 0.1, 17)
    direct = F.point_sources(x, z, e, energy, dist, xp, zp)
    assert F.rel_l2(exact(xp, zp), direct) < 1e-12
