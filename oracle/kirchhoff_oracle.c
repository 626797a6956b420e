/*
 * CPU ORACLE for the Kirchhoff diffraction integral — TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this file's library, and only as the checker or the timed CPU baseline.
 * The product path (xrt-rs_b200/csrc) never calls it.
 *
 * Three restatements of physwkim/xrt-rs algorithms, each written from the
 * reference's published formula in this project's own code:
 *
 *   oracle_kahan_f64   src/waves/diffraction.rs:56-117 (diffraction_integral +
 *                      diffraction_at_pixel): f64, per-component complex Kahan
 *                      summation in ray order, skip path < 1e-30, k = E/CHBAR*1e7.
 *                      The operation order follows the Rust source term for
 *                      term; with -ffp-contract=off and glibc sin/cos every
 *                      per-ray term is computed exactly as Rust computes it.
 *   oracle_plain_f64   src/gpu/fallback.rs:29-71 (kirchhoff_cpu_from_gpu_types):
 *                      f64 plain sum (no Kahan), `* inv_path`, skip < 1e-20.
 *   oracle_kahan_ld    the same formula with the phase k*|p - r| evaluated in
 *                      x87 extended precision (64-bit significand: |p - r| from
 *                      exact differences, sqrtl, sinl/cosl) and everything else
 *                      as oracle_kahan_f64. At 30 keV and 20 m k*path is 3e12
 *                      rad, where one FP64 rounding of the phase is 4.9e-4 rad,
 *                      so the FP64 formula itself carries ~1e-4 relative error
 *                      on noise-like fields; this variant measures that error
 *                      and is the reference for the FP32 phase-reduced path at
 *                      such phases.
 *   oracle_wgsl_f32    src/gpu/shaders/kirchhoff.wgsl:56-135 + the host side in
 *                      src/gpu/kirchhoff.rs:96-297: f32 phase-reduced sum about
 *                      an f32-rounded ray centroid, naive f32 accumulation,
 *                      then the f64 base-phase restore with the mean energy.
 *                      It measures the reference GPU algorithm's own error.
 *
 * And the producers and the sibling sum around the path:
 *
 *   oracle_prepare_wave  src/waves/prepare_wave.rs:40-68 (screen grid, x outer).
 *   oracle_beam_rays     src/waves/prepare_wave.rs:78-111 (beam -> rays, nl = n.dir).
 *   oracle_fresnel       src/waves/fresnel.rs:53-106 (2-D Fresnel sum
 *                        U = sum_j es_j exp(i k/(2d) |p - r_j|^2) over a grid,
 *                        z outer, plain complex accumulation).
 *
 * Pixels run in parallel (OpenMP), mirroring the reference's Rayon
 * `par_iter` over pixels (src/waves/diffraction.rs:60-63); each pixel's ray
 * loop is sequential, so results do not depend on the thread count.
 *
 * Parity pin: oracle_kahan_f64 reproduces the reference fixture
 * validation/fixtures/diffraction_ref.json (5 rays x 3 pixels) to abs 1e-10,
 * the bar of tests/golden_diffraction.rs:119-188.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <omp.h>

/* src/core/consts.rs:74 — c*hbar in eV*Angstrom. */
#define ORACLE_CHBAR 1973.2697177417986
#define ORACLE_PI 3.14159265358979323846

/* Complex helpers mirroring num-complex 0.4 semantics (componentwise add/sub,
 * textbook multiply, no FMA). */
typedef struct { double re, im; } cplx;

static inline cplx c_mul(cplx a, cplx b) {
    cplx r;
    r.re = a.re * b.re - a.im * b.im;
    r.im = a.re * b.im + a.im * b.re;
    return r;
}

static void set_threads(int n_threads) {
    if (n_threads > 0) omp_set_num_threads(n_threads);
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

/* diffraction.rs:67-117, one pixel. */
static void kahan_pixel(const double* rx, const double* ry, const double* rz,
                        const double* rnx, const double* rny, const double* rnz,
                        const double* rnl, const double* es_re, const double* es_im,
                        const double* ep_re, const double* ep_im, const double* energy,
                        size_t n_rays, double px, double py, double pz, double out[4]) {
    cplx es_sum = {0.0, 0.0}, ep_sum = {0.0, 0.0};
    cplx es_comp = {0.0, 0.0}, ep_comp = {0.0, 0.0};
    for (size_t j = 0; j < n_rays; ++j) {
        double dx = px - rx[j];
        double dy = py - ry[j];
        double dz = pz - rz[j];
        double path = sqrt(dx * dx + dy * dy + dz * dz);
        if (path < 1e-30) continue;
        double ns = (rnx[j] * dx + rny[j] * dy + rnz[j] * dz) / path;
        double k = energy[j] / ORACLE_CHBAR * 1e7;
        double phase = k * path;
        double s = sin(phase), c = cos(phase);
        cplx exp_ikr = {c, s};
        double obliquity = rnl[j] + ns;
        double af = k / (4.0 * ORACLE_PI) * obliquity / path;
        /* Complex64::i() * af -> (0*af, 1*af); then * exp_ikr. */
        cplx i_af = {0.0 * af, 1.0 * af};
        cplx u = c_mul(i_af, exp_ikr);

        cplx es = {es_re[j], es_im[j]};
        cplx t = c_mul(es, u);
        cplx es_term = {t.re - es_comp.re, t.im - es_comp.im};
        cplx es_new = {es_sum.re + es_term.re, es_sum.im + es_term.im};
        es_comp.re = (es_new.re - es_sum.re) - es_term.re;
        es_comp.im = (es_new.im - es_sum.im) - es_term.im;
        es_sum = es_new;

        cplx ep = {ep_re[j], ep_im[j]};
        cplx tp = c_mul(ep, u);
        cplx ep_term = {tp.re - ep_comp.re, tp.im - ep_comp.im};
        cplx ep_new = {ep_sum.re + ep_term.re, ep_sum.im + ep_term.im};
        ep_comp.re = (ep_new.re - ep_sum.re) - ep_term.re;
        ep_comp.im = (ep_new.im - ep_sum.im) - ep_term.im;
        ep_sum = ep_new;
    }
    out[0] = es_sum.re; out[1] = es_sum.im; out[2] = ep_sum.re; out[3] = ep_sum.im;
}

/* diffraction.rs:56-64 — pixels in parallel, SoA in, SoA out. */
void oracle_kahan_f64(const double* rx, const double* ry, const double* rz,
                      const double* rnx, const double* rny, const double* rnz,
                      const double* rnl, const double* es_re, const double* es_im,
                      const double* ep_re, const double* ep_im, const double* energy,
                      size_t n_rays, const double* px, const double* py, const double* pz,
                      size_t n_pix, double* o_es_re, double* o_es_im, double* o_ep_re,
                      double* o_ep_im, int n_threads) {
    set_threads(n_threads);
    long long m = (long long)n_pix;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < m; ++i) {
        double o[4];
        kahan_pixel(rx, ry, rz, rnx, rny, rnz, rnl, es_re, es_im, ep_re, ep_im, energy,
                    n_rays, px[i], py[i], pz[i], o);
        o_es_re[i] = o[0]; o_es_im[i] = o[1]; o_ep_re[i] = o[2]; o_ep_im[i] = o[3];
    }
}

/* diffraction.rs:67-117 with an extended-precision phase. */
static void kahan_pixel_ld(const double* rx, const double* ry, const double* rz,
                           const double* rnx, const double* rny, const double* rnz,
                           const double* rnl, const double* es_re, const double* es_im,
                           const double* ep_re, const double* ep_im, const double* energy,
                           size_t n_rays, double px, double py, double pz, double out[4]) {
    cplx es_sum = {0.0, 0.0}, ep_sum = {0.0, 0.0};
    cplx es_comp = {0.0, 0.0}, ep_comp = {0.0, 0.0};
    for (size_t j = 0; j < n_rays; ++j) {
        double dx = px - rx[j];
        double dy = py - ry[j];
        double dz = pz - rz[j];
        double path = sqrt(dx * dx + dy * dy + dz * dz);
        if (path < 1e-30) continue;
        double ns = (rnx[j] * dx + rny[j] * dy + rnz[j] * dz) / path;
        double k = energy[j] / ORACLE_CHBAR * 1e7;
        long double lx = (long double)px - (long double)rx[j];
        long double ly = (long double)py - (long double)ry[j];
        long double lz = (long double)pz - (long double)rz[j];
        long double phase = (long double)k * sqrtl(lx * lx + ly * ly + lz * lz);
        cplx exp_ikr = {(double)cosl(phase), (double)sinl(phase)};
        double obliquity = rnl[j] + ns;
        double af = k / (4.0 * ORACLE_PI) * obliquity / path;
        cplx i_af = {0.0 * af, 1.0 * af};
        cplx u = c_mul(i_af, exp_ikr);

        cplx es = {es_re[j], es_im[j]};
        cplx t = c_mul(es, u);
        cplx es_term = {t.re - es_comp.re, t.im - es_comp.im};
        cplx es_new = {es_sum.re + es_term.re, es_sum.im + es_term.im};
        es_comp.re = (es_new.re - es_sum.re) - es_term.re;
        es_comp.im = (es_new.im - es_sum.im) - es_term.im;
        es_sum = es_new;

        cplx ep = {ep_re[j], ep_im[j]};
        cplx tp = c_mul(ep, u);
        cplx ep_term = {tp.re - ep_comp.re, tp.im - ep_comp.im};
        cplx ep_new = {ep_sum.re + ep_term.re, ep_sum.im + ep_term.im};
        ep_comp.re = (ep_new.re - ep_sum.re) - ep_term.re;
        ep_comp.im = (ep_new.im - ep_sum.im) - ep_term.im;
        ep_sum = ep_new;
    }
    out[0] = es_sum.re; out[1] = es_sum.im; out[2] = ep_sum.re; out[3] = ep_sum.im;
}

void oracle_kahan_ld(const double* rx, const double* ry, const double* rz,
                     const double* rnx, const double* rny, const double* rnz,
                     const double* rnl, const double* es_re, const double* es_im,
                     const double* ep_re, const double* ep_im, const double* energy,
                     size_t n_rays, const double* px, const double* py, const double* pz,
                     size_t n_pix, double* o_es_re, double* o_es_im, double* o_ep_re,
                     double* o_ep_im, int n_threads) {
    set_threads(n_threads);
    long long m = (long long)n_pix;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < m; ++i) {
        double o[4];
        kahan_pixel_ld(rx, ry, rz, rnx, rny, rnz, rnl, es_re, es_im, ep_re, ep_im, energy,
                       n_rays, px[i], py[i], pz[i], o);
        o_es_re[i] = o[0]; o_es_im[i] = o[1]; o_ep_re[i] = o[2]; o_ep_im[i] = o[3];
    }
}

/* fallback.rs:29-71 — plain f64 sum over f32 inputs promoted to f64. The
 * caller passes f64 arrays holding the f32-rounded values. */
void oracle_plain_f64(const double* rx, const double* ry, const double* rz,
                      const double* rnx, const double* rny, const double* rnz,
                      const double* rnl, const double* es_re, const double* es_im,
                      const double* ep_re, const double* ep_im, const double* energy,
                      size_t n_rays, const double* px, const double* py, const double* pz,
                      size_t n_pix, double* o_es_re, double* o_es_im, double* o_ep_re,
                      double* o_ep_im, int n_threads) {
    set_threads(n_threads);
    long long m = (long long)n_pix;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < m; ++i) {
        cplx es = {0.0, 0.0}, ep = {0.0, 0.0};
        for (size_t j = 0; j < n_rays; ++j) {
            double dx = px[i] - rx[j];
            double dy = py[i] - ry[j];
            double dz = pz[i] - rz[j];
            double path = sqrt(dx * dx + dy * dy + dz * dz);
            if (path < 1e-20) continue;
            double inv_path = 1.0 / path;
            double ns = (rnx[j] * dx + rny[j] * dy + rnz[j] * dz) * inv_path;
            double k = energy[j] / ORACLE_CHBAR * 1e7;
            double phase = k * path;
            double s = sin(phase), c = cos(phase);
            double obliquity = rnl[j] + ns;
            double amp = k / (4.0 * ORACLE_PI) * obliquity * inv_path;
            cplx u = {-amp * s, amp * c};
            cplx a = {es_re[j], es_im[j]}, b = {ep_re[j], ep_im[j]};
            cplx ta = c_mul(a, u), tb = c_mul(b, u);
            es.re += ta.re; es.im += ta.im;
            ep.re += tb.re; ep.im += tb.im;
        }
        o_es_re[i] = es.re; o_es_im[i] = es.im; o_ep_re[i] = ep.re; o_ep_im[i] = ep.im;
    }
}

/* kirchhoff.wgsl:56-135 (device, f32) + kirchhoff.rs:96-115,276-297 (host).
 * Inputs are f32 arrays (the GpuRay / GpuPixel fields). */
void oracle_wgsl_f32(const float* rx, const float* ry, const float* rz,
                     const float* rnx, const float* rny, const float* rnz,
                     const float* rnl, const float* energy,
                     const float* es_re, const float* es_im,
                     const float* ep_re, const float* ep_im, size_t n_rays,
                     const float* px, const float* py, const float* pz, size_t n_pix,
                     double* o_es_re, double* o_es_im, double* o_ep_re, double* o_ep_im,
                     int n_threads) {
    set_threads(n_threads);
    /* kirchhoff.rs:96-104: f64 centroid and mean energy over the f32 rays. */
    double n = (double)n_rays;
    double sx = 0.0, sy = 0.0, sz = 0.0, se = 0.0;
    for (size_t j = 0; j < n_rays; ++j) { sx += (double)rx[j]; }
    for (size_t j = 0; j < n_rays; ++j) { sy += (double)ry[j]; }
    for (size_t j = 0; j < n_rays; ++j) { sz += (double)rz[j]; }
    for (size_t j = 0; j < n_rays; ++j) { se += (double)energy[j]; }
    double cx64 = sx / n, cy64 = sy / n, cz64 = sz / n;
    double k64 = (se / n) / ORACLE_CHBAR * 1e7;
    /* GpuParams (kirchhoff.rs:106-115): f32-rounded centroid and 1/CHBAR*1e7. */
    float cx = (float)cx64, cy = (float)cy64, cz = (float)cz64;
    float chbar_inv_1e7 = (float)(1.0 / ORACLE_CHBAR * 1e7);
    const float PI_F = 3.14159265358979323846f;
    long long m = (long long)n_pix;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < m; ++i) {
        float pxi = px[i], pyi = py[i], pzi = pz[i];
        float rdx = pxi - cx, rdy = pyi - cy, rdz = pzi - cz;
        float ref_path = sqrtf(rdx * rdx + rdy * rdy + rdz * rdz);
        float a_re = 0.f, a_im = 0.f, b_re = 0.f, b_im = 0.f;
        for (size_t j = 0; j < n_rays; ++j) {
            float dx = pxi - rx[j], dy = pyi - ry[j], dz = pzi - rz[j];
            float path = sqrtf(dx * dx + dy * dy + dz * dz);
            if (path < 1e-20f) continue;
            float inv_path = 1.0f / path;
            float ns = (rnx[j] * dx + rny[j] * dy + rnz[j] * dz) * inv_path;
            float k = energy[j] * chbar_inv_1e7;
            float ox = cx - rx[j], oy = cy - ry[j], oz = cz - rz[j];
            float diff_sq = ox * (2.0f * pxi - cx - rx[j]) + oy * (2.0f * pyi - cy - ry[j]) +
                            oz * (2.0f * pzi - cz - rz[j]);
            float delta_path = diff_sq / (path + ref_path);
            float dphi = k * delta_path;
            float c = cosf(dphi), s = sinf(dphi);
            float obl = rnl[j] + ns;
            float amp = k / (4.0f * PI_F) * obl * inv_path;
            float u_re = -amp * s, u_im = amp * c;
            a_re += es_re[j] * u_re - es_im[j] * u_im;
            a_im += es_re[j] * u_im + es_im[j] * u_re;
            b_re += ep_re[j] * u_re - ep_im[j] * u_im;
            b_im += ep_re[j] * u_im + ep_im[j] * u_re;
        }
        /* kirchhoff.rs:278-297: restore exp(i*k_mean*|p - c64|) in f64. */
        double dx = (double)pxi - cx64, dy = (double)pyi - cy64, dz = (double)pzi - cz64;
        double refp = sqrt(dx * dx + dy * dy + dz * dz);
        double bp = k64 * refp;
        double sb = sin(bp), cb = cos(bp);
        cplx ph = {cb, sb};
        cplx es = {(double)a_re, (double)a_im}, ep = {(double)b_re, (double)b_im};
        cplx r1 = c_mul(es, ph), r2 = c_mul(ep, ph);
        o_es_re[i] = r1.re; o_es_im[i] = r1.im; o_ep_re[i] = r2.re; o_ep_im[i] = r2.im;
    }
}


/* ---- screen grid (src/waves/prepare_wave.rs:40-68) ---------------------- */

static double grid_frac(size_t i, size_t n) {
    return n > 1 ? (double)i / (double)(n - 1) - 0.5 : 0.0;
}

void oracle_prepare_wave(const double* center, double dx, double dz, size_t nx, size_t nz,
                         double* px, double* py, double* pz) {
    for (size_t ix = 0; ix < nx; ++ix) {
        double x = center[0] + grid_frac(ix, nx) * 2.0 * dx;
        for (size_t iz = 0; iz < nz; ++iz) {
            size_t i = ix * nz + iz;
            px[i] = x;
            py[i] = center[1];
            pz[i] = center[2] + grid_frac(iz, nz) * 2.0 * dz;
        }
    }
}

/* ---- beam -> rays (src/waves/prepare_wave.rs:78-111) --------------------
 * beam: 7 columns (x, y, z, a, b, c, e) then 4 amplitude columns or NULLs;
 * normals: n_beam rows of 3; out: the 12 ray columns. */
void oracle_beam_rays(const double* const* beam, const double* normals, const size_t* good,
                      size_t n_good, double* const* out) {
    for (size_t i = 0; i < n_good; ++i) {
        size_t j = good[i];
        const double* n = normals + 3 * j;
        out[0][i] = beam[0][j];
        out[1][i] = beam[1][j];
        out[2][i] = beam[2][j];
        out[3][i] = n[0];
        out[4][i] = n[1];
        out[5][i] = n[2];
        out[6][i] = n[0] * beam[3][j] + n[1] * beam[4][j] + n[2] * beam[5][j];
        if (beam[7]) {
            out[7][i] = beam[7][j];
            out[8][i] = beam[8][j];
            out[9][i] = beam[9][j];
            out[10][i] = beam[10][j];
        } else {
            out[7][i] = 1.0;
            out[8][i] = 0.0;
            out[9][i] = 0.0;
            out[10][i] = 0.0;
        }
        out[11][i] = beam[6][j];
    }
}

/* ---- 2-D Fresnel sum (src/waves/fresnel.rs:53-106) ----------------------
 * Screen coordinates x_i = x_min + (x_max - x_min) * i / max(nx - 1, 1)
 * (same for z); output index iz * nx + ix; per term
 * es_j * exp((0, k/(2d)) * r2) with the complex exponential of a purely
 * imaginary argument (cos, sin), textbook complex multiply, plain sum. */
void oracle_fresnel(const double* rx, const double* rz, const double* es_re, const double* es_im,
                    size_t n, double energy, double dist, double x_min, double x_max, size_t nx,
                    double z_min, double z_max, size_t nz, double* o_re, double* o_im,
                    int n_threads) {
    set_threads(n_threads);
    const double k = energy / ORACLE_CHBAR * 1e7;
    const double pre_im = k / (2.0 * dist);
    const double xden = (double)(nx > 1 ? nx - 1 : 1), zden = (double)(nz > 1 ? nz - 1 : 1);
    long long total = (long long)(nx * nz);
#pragma omp parallel for schedule(dynamic, 16)
    for (long long idx = 0; idx < total; ++idx) {
        size_t iz = (size_t)idx / nx, ix = (size_t)idx - iz * nx;
        double xp = x_min + (x_max - x_min) * (double)ix / xden;
        double zp = z_min + (z_max - z_min) * (double)iz / zden;
        double s_re = 0.0, s_im = 0.0;
        for (size_t j = 0; j < n; ++j) {
            double dx = xp - rx[j];
            double dz = zp - rz[j];
            double r2 = dx * dx + dz * dz;
            double th = pre_im * r2;
            cplx ph = {cos(th), sin(th)};
            cplx e = {es_re[j], es_im[j]};
            cplx t = c_mul(e, ph);
            s_re += t.re;
            s_im += t.im;
        }
        o_re[idx] = s_re;
        o_im[idx] = s_im;
    }
}
