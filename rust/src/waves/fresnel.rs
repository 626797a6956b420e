//! 2D Fresnel wavefront propagation on the sm_100a engine (libxk.so).
//!
//! U(x, z) = sum_j es_j exp(i k/(2 dist) ((x - x_j)^2 + (z - z_j)^2)) on a
//! regular nx x nz screen, output index iz * nx + ix. `fresnel_propagate`
//! keeps its signature and runs the library's FP64 sum (term for term, the
//! parity path); `fresnel_propagate_separable` runs the tensor-core
//! separable product (relative L2 <= 1e-4 of the FP64 sum).

use num_complex::Complex64;

use crate::gpu::context::GpuContext;
use crate::gpu::xk_ffi;

/// Observation screen configuration for Fresnel propagation.
pub struct FresnelScreen {
    /// X range minimum [mm]
    pub x_min: f64,
    /// X range maximum [mm]
    pub x_max: f64,
    /// Number of x pixels
    pub nx: usize,
    /// Z range minimum [mm]
    pub z_min: f64,
    /// Z range maximum [mm]
    pub z_max: f64,
    /// Number of z pixels
    pub nz: usize,
}

/// Result of Fresnel propagation.
pub struct FresnelResult {
    /// Complex amplitude at each observation pixel
    pub amplitude: Vec<Complex64>,
    /// Pixel x-coordinates [mm]
    pub x_pixels: Vec<f64>,
    /// Pixel z-coordinates [mm]
    pub z_pixels: Vec<f64>,
    /// Number of x pixels
    pub nx: usize,
    /// Number of z pixels
    pub nz: usize,
}

impl FresnelResult {
    /// Compute intensity at each pixel.
    pub fn intensity(&self) -> Vec<f64> {
        self.amplitude.iter().map(|a| a.norm_sqr()).collect()
    }
}

/// Perform 2D Fresnel propagation from source rays at z = 0 to an
/// observation screen at distance `dist` (FP64 sum on the GPU).
pub fn fresnel_propagate(
    ray_x: &[f64],
    ray_z: &[f64],
    ray_es: &[Complex64],
    energy: f64,
    dist: f64,
    screen: &FresnelScreen,
) -> FresnelResult {
    propagate(ray_x, ray_z, ray_es, energy, dist, screen, xk_ffi::XK_PATH_F64)
}

/// The same propagation as one complex matrix product on the tensor cores.
pub fn fresnel_propagate_separable(
    ray_x: &[f64],
    ray_z: &[f64],
    ray_es: &[Complex64],
    energy: f64,
    dist: f64,
    screen: &FresnelScreen,
) -> FresnelResult {
    propagate(ray_x, ray_z, ray_es, energy, dist, screen, xk_ffi::XK_PATH_SEPARABLE)
}

fn propagate(
    ray_x: &[f64],
    ray_z: &[f64],
    ray_es: &[Complex64],
    energy: f64,
    dist: f64,
    screen: &FresnelScreen,
    path: i32,
) -> FresnelResult {
    let n = ray_x.len();
    assert!(ray_z.len() == n && ray_es.len() == n, "ray arrays differ in length");
    let es_re: Vec<f64> = ray_es.iter().map(|c| c.re).collect();
    let es_im: Vec<f64> = ray_es.iter().map(|c| c.im).collect();
    let m = screen.nx * screen.nz;
    let (mut re, mut im) = (vec![0.0; m], vec![0.0; m]);
    let mut xp = vec![0.0; screen.nx];
    let mut zp = vec![0.0; screen.nz];
    if m > 0 {
        let ctx = GpuContext::shared().expect("fresnel_propagate: no CUDA device");
        let sc = xk_ffi::xk_fresnel_screen {
            x_min: screen.x_min,
            x_max: screen.x_max,
            nx: screen.nx,
            z_min: screen.z_min,
            z_max: screen.z_max,
            nz: screen.nz,
        };
        let rc = unsafe {
            xk_ffi::xk_fresnel_propagate(ctx.raw(), ray_x.as_ptr(), ray_z.as_ptr(),
                                         es_re.as_ptr(), es_im.as_ptr(), n, energy, dist, &sc,
                                         re.as_mut_ptr(), im.as_mut_ptr(), xp.as_mut_ptr(),
                                         zp.as_mut_ptr(), path, std::ptr::null_mut())
        };
        xk_ffi::check(rc, ctx.raw(), "xk_fresnel_propagate");
    } else {
        // Empty screen: no launch, coordinates from the screen formula.
        let grid = |lo: f64, hi: f64, k: usize, out: &mut Vec<f64>| {
            let den = if k > 1 { (k - 1) as f64 } else { 1.0 };
            for (i, v) in out.iter_mut().enumerate() {
                *v = lo + (hi - lo) * i as f64 / den;
            }
        };
        grid(screen.x_min, screen.x_max, screen.nx, &mut xp);
        grid(screen.z_min, screen.z_max, screen.nz, &mut zp);
    }
    FresnelResult {
        amplitude: re.iter().zip(&im).map(|(&r, &i)| Complex64::new(r, i)).collect(),
        x_pixels: xp,
        z_pixels: zp,
        nx: screen.nx,
        nz: screen.nz,
    }
}
