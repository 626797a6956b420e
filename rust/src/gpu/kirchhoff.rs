//! GPU Kirchhoff diffraction integral on the sm_100a engine (libxk.so).
//!
//! `kirchhoff_gpu` keeps its signature and record types. The records go to
//! the device as they are (48-byte rays, 16-byte pixels), are widened to f64
//! there, and the FP32 phase-reduced solve runs with its base phases in FP64;
//! the field comes back as four f64 per pixel.

use bytemuck::{Pod, Zeroable};
use num_complex::Complex64;

use crate::gpu::context::GpuContext;
use crate::gpu::xk_ffi;

/// GPU-compatible ray data (f32, 48 bytes).
#[repr(C)]
#[derive(Debug, Clone, Copy, Pod, Zeroable)]
pub struct GpuRay {
    pub x: f32,
    pub y: f32,
    pub z: f32,
    pub nx: f32,
    pub ny: f32,
    pub nz: f32,
    pub nl: f32,
    pub energy: f32,
    pub es_re: f32,
    pub es_im: f32,
    pub ep_re: f32,
    pub ep_im: f32,
}

/// GPU-compatible pixel position (16 bytes).
#[repr(C)]
#[derive(Debug, Clone, Copy, Pod, Zeroable)]
pub struct GpuPixel {
    pub x: f32,
    pub y: f32,
    pub z: f32,
    pub _pad: f32,
}

/// GPU-compatible result (16 bytes).
#[repr(C)]
#[derive(Debug, Clone, Copy, Pod, Zeroable)]
pub struct GpuPixelResult {
    pub es_re: f32,
    pub es_im: f32,
    pub ep_re: f32,
    pub ep_im: f32,
}

const _: () = assert!(std::mem::size_of::<GpuRay>() == 48);
const _: () = assert!(std::mem::size_of::<GpuPixel>() == 16);

/// The four doubles per pixel that `xk_kirchhoff_gpu` writes, in C order
/// (a tuple's layout is not guaranteed, so the field goes through this).
#[repr(C)]
#[derive(Clone, Copy, Default)]
pub(crate) struct FieldRecord {
    pub es_re: f64,
    pub es_im: f64,
    pub ep_re: f64,
    pub ep_im: f64,
}

impl FieldRecord {
    pub(crate) fn pair(self) -> (Complex64, Complex64) {
        (Complex64::new(self.es_re, self.es_im), Complex64::new(self.ep_re, self.ep_im))
    }
}

/// Run the Kirchhoff diffraction integral on the GPU. Returns the complex
/// field amplitudes (Es, Ep) per pixel, in pixel order. Panics if the
/// library reports an error.
pub fn kirchhoff_gpu(
    ctx: &GpuContext,
    rays: &[GpuRay],
    pixels: &[GpuPixel],
) -> Vec<(Complex64, Complex64)> {
    let mut out = vec![FieldRecord::default(); pixels.len()];
    let rc = unsafe {
        xk_ffi::xk_kirchhoff_gpu(
            ctx.raw(),
            rays.as_ptr(),
            rays.len(),
            pixels.as_ptr(),
            pixels.len(),
            out.as_mut_ptr() as *mut f64,
        )
    };
    xk_ffi::check(rc, ctx.raw(), "xk_kirchhoff_gpu");
    out.into_iter().map(FieldRecord::pair).collect()
}
