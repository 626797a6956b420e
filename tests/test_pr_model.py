"""CPU check of the FP32 phase-reduced decomposition (no GPU).

Restates, in float64 numpy, the per-pair algebra the persistent kernel uses
(xrt-rs_b200/csrc/xk_pr.cu): per-chunk centre R0, per-tile direction u,
residual k*Delta = k(|rho_perp|^2 - 2 v.rho)/(2(|q| - u.rho)), the series
reciprocal of the packed sweep, the obliquity from 2n.(q - rho), and the
FP64 phasors exp(i k|q|) and exp(-i k u.rho). In float64 the decomposition is
exact up to the neglected Delta/|q| and e^3 terms — k Delta^2 / (2|q|) rad,
under 1e-6 rad while |k Delta| stays within a ~300 rad budget. What remains
is FP64 itself: k|q| ~ 5e10 rad is rounded once per (screen point, chunk),
an error of up to ulp/2 = 3.8e-6 rad shared by the whole chunk, where the
oracle rounds k*path per term and those errors average out. So the model
must reproduce the oracle to ~1e-5 — a check of the formulas, signs and
factors, independent of the GPU.
"""
import numpy as np
import pytest

import cases
from xrt_rs import synth


def model(rays, pix, chunk_cells=24, series=False, max_phase=300.0):
    k = synth.wavenumber(rays["energy"][0])
    kt = k / (2 * np.pi)
    r = np.stack([rays["x"], rays["y"], rays["z"]], 1)
    n = np.stack([rays["nx"], rays["ny"], rays["nz"]], 1)
    es = rays["es_re"] + 1j * rays["es_im"]
    ep = rays["ep_re"] + 1j * rays["ep_im"]
    p = np.stack([pix["x"], pix["y"], pix["z"]], 1)
    P0 = 0.5 * (p.min(0) + p.max(0))
    # Chunks: a coarse grid over the transverse plane, centre = cell centre.
    lo, hi = r.min(0), r.max(0)
    h = np.maximum((hi - lo) / chunk_cells, 1e-12)
    cell = np.floor((r - lo) / h).clip(0, chunk_cells - 1)
    key = cell[:, 0] * chunk_cells * chunk_cells + cell[:, 1] * chunk_cells + cell[:, 2]
    out_es = np.zeros(len(p), complex)
    out_ep = np.zeros(len(p), complex)
    for kk in np.unique(key):
        sel = key == kk
        R0 = lo + (cell[sel][0] + 0.5) * h
        rho = r[sel] - R0
        D = P0 - R0
        u = D / np.linalg.norm(D)
        ur = rho @ u
        perp2 = np.sum((rho - ur[:, None] * u) ** 2, 1)
        q = p - R0
        qn = np.linalg.norm(q, axis=1)
        v = q - qn[:, None] * u
        num = k * (perp2[None, :] - 2 * (v @ rho.T))
        if series:
            r0 = 0.5 / qn[:, None]
            e = 2 * ur[None, :] * r0
            rd = r0 * (1 + e + e * e)
        else:
            rd = 1.0 / (2 * qn[:, None] - 2 * ur[None, :])
        th = num * rd
        # The kernel's denominator drops Delta; that is only negligible while
        # the residual phase stays within the planner's budget.
        assert np.abs(th).max() <= max_phase
        g = 2 * (q @ n[sel].T) - 2 * np.sum(n[sel] * rho, 1)[None, :]
        obl = rays["nl"][sel][None, :] + g * rd
        amp = obl * rd
        ray_ph = np.exp(-1j * k * ur)
        pix_ph = kt * 1j * np.exp(1j * k * qn)
        term = amp * np.exp(1j * th)
        out_es += pix_ph * (term @ (es[sel] * ray_ph))
        out_ep += pix_ph * (term @ (ep[sel] * ray_ph))
    return out_es.real, out_es.imag, out_ep.real, out_ep.imag


@pytest.mark.parametrize("series", [False, True])
def test_decomposition_matches_oracle_config0(oracle, series):
    rays, pix = synth.config0(seed=2)
    ref = oracle.kahan_f64(*cases.as_lists(rays, pix))
    out = model(rays, pix, series=series)
    assert cases.rel_l2(out, ref) < 2e-5


def test_decomposition_general_normals(oracle):
    rays, pix = cases.random_case(400, 50, seed=4, general_normals=True)
    ref = oracle.kahan_f64(*cases.as_lists(rays, pix))
    out = model(rays, pix)
    assert cases.rel_l2(out, ref) < 2e-5
