//! Auto dispatch of the GPU Kirchhoff integral.
//!
//! On this engine there is no CPU fallback: `kirchhoff_auto` runs on the
//! shared CUDA context and panics when no device exists, instead of running
//! an f64 loop on the host.

use num_complex::Complex64;

use crate::gpu::kirchhoff::{FieldRecord, GpuPixel, GpuRay};
use crate::gpu::xk_ffi;

/// Kirchhoff diffraction on the shared GPU context. Returns (Es, Ep) per
/// pixel, same as `kirchhoff_gpu`; panics with XK_ERR_NO_DEVICE when there is
/// no CUDA device.
pub fn kirchhoff_auto(rays: &[GpuRay], pixels: &[GpuPixel]) -> Vec<(Complex64, Complex64)> {
    let mut out = vec![FieldRecord::default(); pixels.len()];
    let rc = unsafe {
        xk_ffi::xk_kirchhoff_auto(
            rays.as_ptr(),
            rays.len(),
            pixels.as_ptr(),
            pixels.len(),
            out.as_mut_ptr() as *mut f64,
        )
    };
    xk_ffi::check(rc, std::ptr::null(), "xk_kirchhoff_auto");
    out.into_iter().map(FieldRecord::pair).collect()
}
