"""Closed-form 2-D Fresnel fields that pin the Fresnel sum independently of its
implementation (src/waves/fresnel.rs:53-106 sums
U(x, z) = sum_j es_j exp(i a ((x - x_j)^2 + (z - z_j)^2)), a = k / (2 d)).

* one point source:   U = es exp(i a r^2);
* two point sources:  the sum of two such terms;
* a row of N equal rays at the Talbot pitch h = sqrt(2 pi m / a) along x:
  a (j h)^2 is a multiple of 2 pi, so with t = x - x0
      U = es exp(i a (t^2 + (z - z0)^2)) sum_{j<N} exp(-2 i a t h j)
        = es exp(i a (t^2 + (z - z0)^2)) exp(-i (N - 1) s) sin(N s) / sin(s),
  s = a t h — a geometric series evaluated in closed form, not term by term.

Phases are formed and reduced modulo 2 pi in extended precision (numpy
longdouble), so the values are exact to ~1e-15 relative. Screen coordinates
follow the reference's grid x_i = x_min + (x_max - x_min) i / max(nx - 1, 1),
output index iz * nx + ix (src/waves/fresnel.rs:60-75).
"""
import numpy as np

CHBAR = np.longdouble("1973.2697177417986")  # src/core/consts.rs:74
TWO_PI = 2 * np.longdouble("3.14159265358979323846264338327950288")


def a_coef(energy, dist):
    """a = k / (2 d) in extended precision, k = E / CHBAR * 1e7 [1/mm]."""
    k = np.longdouble(energy) / CHBAR * np.longdouble(1e7)
    return k / (2 * np.longdouble(dist))


def screen_coords(x_min, x_max, nx, z_min, z_max, nz):
    xs = x_min + (x_max - x_min) * np.arange(nx, dtype=np.float64) / float(max(nx - 1, 1))
    zs = z_min + (z_max - z_min) * np.arange(nz, dtype=np.float64) / float(max(nz - 1, 1))
    zp, xp = np.meshgrid(zs, xs, indexing="ij")
    return xp.reshape(-1), zp.reshape(-1)


def _cis(phase_ld):
    red = np.mod(phase_ld, TWO_PI)
    return np.exp(1j * np.asarray(red, dtype=np.float64))


def point_sources(xs, zs, es, energy, dist, xp, zp):
    """Sum of len(xs) point-source terms, each evaluated exactly."""
    a = a_coef(energy, dist)
    out = np.zeros(len(xp), dtype=np.complex128)
    for x0, z0, e in zip(xs, zs, es):
        dx = np.asarray(xp, dtype=np.longdouble) - np.longdouble(x0)
        dz = np.asarray(zp, dtype=np.longdouble) - np.longdouble(z0)
        out += complex(e) * _cis(a * (dx * dx + dz * dz))
    return out


def talbot_pitch(energy, dist, m=1):
    """Pitch h (float64) with a h^2 = 2 pi m."""
    return float(np.sqrt(TWO_PI * m / a_coef(energy, dist)))


def talbot_row(n, x0, z0, es, energy, dist, m=1):
    """Rays (x, z, es arrays) of the Talbot row and its closed-form field
    function f(xp, zp)."""
    h = talbot_pitch(energy, dist, m)
    x = x0 + h * np.arange(n, dtype=np.float64)
    z = np.full(n, float(z0))
    e = np.full(n, complex(es))
    a = a_coef(energy, dist)
    hl = np.sqrt(TWO_PI * m / a)

    def field(xp, zp):
        t = np.asarray(xp, dtype=np.longdouble) - np.longdouble(x0)
        dz = np.asarray(zp, dtype=np.longdouble) - np.longdouble(z0)
        s = a * t * hl  # half the phase step of the series
        base = _cis(a * (t * t + dz * dz) - (n - 1) * s)
        # sin(N s) / sin(s), its limit +-N where sin(s) = 0
        num = np.sin(np.mod(n * s, TWO_PI))  # extended precision (sinl)
        den = np.sin(np.mod(s, TWO_PI))
        ratio = np.empty(len(t))
        small = np.abs(den) < 1e-15
        ratio[~small] = np.asarray(num[~small] / den[~small], dtype=np.float64)
        # near s = pi q: sin(N s)/sin(s) -> N cos(pi q N)/cos(pi q) = N (-1)^(q (N - 1))
        q = np.rint(np.asarray(s / (TWO_PI / 2), dtype=np.float64))
        ratio[small] = n * np.where((q[small] * (n - 1)) % 2 == 0, 1.0, -1.0)
        return complex(es) * base * ratio

    return x, z, e, field


def rel_l2(got, ref):
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
