//! Kirchhoff diffraction integral on the sm_100a engine (libxk.so).
//!
//! For each pixel, sums over all rays on the OE
//!   U = (k i)/(4 pi) (nl + ns) exp(i k path) / path,
//!   Es += es_j U,  Ep += ep_j U,
//! skipping rays within 1e-30 mm of the pixel. `diffraction_integral` keeps
//! its signature and runs the library's FP64 path, the same per-pair
//! arithmetic with per-component Kahan sums in ray order (<= 1e-10 relative
//! L2 from the f64 CPU loop); `diffraction_integral_with` selects the FP32
//! phase-reduced path (<= 1e-4) or a private context.

use num_complex::Complex64;

use crate::gpu::context::GpuContext;
use crate::gpu::xk_ffi;

/// A single ray on the OE surface, ready for diffraction computation.
#[derive(Debug, Clone, Copy)]
pub struct DiffractionRay {
    /// Position on the OE [mm]
    pub x: f64,
    pub y: f64,
    pub z: f64,
    /// Surface normal at ray position
    pub nx: f64,
    pub ny: f64,
    pub nz: f64,
    /// Obliquity factor (local_n . beam_direction)
    pub nl: f64,
    /// Field amplitudes
    pub es: Complex64,
    pub ep: Complex64,
    /// Energy [eV]
    pub energy: f64,
}

/// A pixel in the observation plane.
#[derive(Debug, Clone, Copy)]
pub struct PixelPoint {
    pub x: f64,
    pub y: f64,
    pub z: f64,
}

/// Result of diffraction at a single pixel.
#[derive(Debug, Clone, Copy)]
pub struct DiffractionResult {
    pub es: Complex64,
    pub ep: Complex64,
}

/// Which of the library's forms computes the sum.
#[derive(Debug, Clone, Copy, PartialEq, Eq)]
pub enum KirchhoffPath {
    /// The reference arithmetic in FP64 (parity path).
    F64,
    /// FP32 phase-reduced form (relative L2 <= 1e-4 for E <= 30 keV, d <= 20 m).
    F32PhaseReduced,
}

/// Compute the Kirchhoff diffraction integral. Returns one
/// `DiffractionResult` per pixel, in pixel order. Panics without a CUDA
/// device (there is no CPU fallback).
pub fn diffraction_integral(
    rays: &[DiffractionRay],
    pixels: &[PixelPoint],
) -> Vec<DiffractionResult> {
    let ctx = GpuContext::shared().expect("diffraction_integral: no CUDA device");
    diffraction_integral_with(ctx, rays, pixels, KirchhoffPath::F64)
}

/// The integral on a given context and path.
pub fn diffraction_integral_with(
    ctx: &GpuContext,
    rays: &[DiffractionRay],
    pixels: &[PixelPoint],
    path: KirchhoffPath,
) -> Vec<DiffractionResult> {
    let cols = RayColumns::from_rays(rays);
    let px: Vec<f64> = pixels.iter().map(|p| p.x).collect();
    let py: Vec<f64> = pixels.iter().map(|p| p.y).collect();
    let pz: Vec<f64> = pixels.iter().map(|p| p.z).collect();
    let (es_re, es_im, ep_re, ep_im) = solve_columns(ctx, &cols, &px, &py, &pz, path);
    (0..pixels.len())
        .map(|i| DiffractionResult {
            es: Complex64::new(es_re[i], es_im[i]),
            ep: Complex64::new(ep_re[i], ep_im[i]),
        })
        .collect()
}

/// Ray columns in the library's structure-of-arrays layout.
pub(crate) struct RayColumns {
    pub x: Vec<f64>,
    pub y: Vec<f64>,
    pub z: Vec<f64>,
    pub nx: Vec<f64>,
    pub ny: Vec<f64>,
    pub nz: Vec<f64>,
    pub nl: Vec<f64>,
    pub es_re: Vec<f64>,
    pub es_im: Vec<f64>,
    pub ep_re: Vec<f64>,
    pub ep_im: Vec<f64>,
    pub energy: Vec<f64>,
}

impl RayColumns {
    pub(crate) fn from_rays(rays: &[DiffractionRay]) -> Self {
        let col = |f: &dyn Fn(&DiffractionRay) -> f64| rays.iter().map(f).collect::<Vec<f64>>();
        Self {
            x: col(&|r| r.x),
            y: col(&|r| r.y),
            z: col(&|r| r.z),
            nx: col(&|r| r.nx),
            ny: col(&|r| r.ny),
            nz: col(&|r| r.nz),
            nl: col(&|r| r.nl),
            es_re: col(&|r| r.es.re),
            es_im: col(&|r| r.es.im),
            ep_re: col(&|r| r.ep.re),
            ep_im: col(&|r| r.ep.im),
            energy: col(&|r| r.energy),
        }
    }

    pub(crate) fn len(&self) -> usize {
        self.x.len()
    }

    pub(crate) fn ffi(&self) -> xk_ffi::xk_rays {
        xk_ffi::xk_rays {
            x: self.x.as_ptr(),
            y: self.y.as_ptr(),
            z: self.z.as_ptr(),
            nx: self.nx.as_ptr(),
            ny: self.ny.as_ptr(),
            nz: self.nz.as_ptr(),
            nl: self.nl.as_ptr(),
            es_re: self.es_re.as_ptr(),
            es_im: self.es_im.as_ptr(),
            ep_re: self.ep_re.as_ptr(),
            ep_im: self.ep_im.as_ptr(),
            energy: self.energy.as_ptr(),
        }
    }
}

/// One solve through `xk_diffraction_integral` on host columns; returns
/// (es_re, es_im, ep_re, ep_im).
pub(crate) fn solve_columns(
    ctx: &GpuContext,
    rays: &RayColumns,
    px: &[f64],
    py: &[f64],
    pz: &[f64],
    path: KirchhoffPath,
) -> (Vec<f64>, Vec<f64>, Vec<f64>, Vec<f64>) {
    let m = px.len();
    assert!(py.len() == m && pz.len() == m, "pixel columns differ in length");
    let mut out = (vec![0.0; m], vec![0.0; m], vec![0.0; m], vec![0.0; m]);
    if m == 0 {
        return out;
    }
    let r = rays.ffi();
    let p = xk_ffi::xk_pixels { x: px.as_ptr(), y: py.as_ptr(), z: pz.as_ptr() };
    let mut f = xk_ffi::xk_field {
        es_re: out.0.as_mut_ptr(),
        es_im: out.1.as_mut_ptr(),
        ep_re: out.2.as_mut_ptr(),
        ep_im: out.3.as_mut_ptr(),
    };
    let code = match path {
        KirchhoffPath::F64 => xk_ffi::XK_PATH_F64,
        KirchhoffPath::F32PhaseReduced => xk_ffi::XK_PATH_F32PR,
    };
    let rc = unsafe {
        xk_ffi::xk_diffraction_integral(ctx.raw(), &r, rays.len(), &p, m, &mut f, code,
                                        std::ptr::null_mut())
    };
    xk_ffi::check(rc, ctx.raw(), "xk_diffraction_integral");
    out
}
