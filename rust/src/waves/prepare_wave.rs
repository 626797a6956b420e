//! Wave preparation on the device: the screen grid and the beam-to-ray
//! conversion in front of the Kirchhoff integral, with the reference's
//! operation order (results are bit-identical to the f64 CPU loops).

use num_complex::Complex64;

use crate::core::beam::Beam;
use crate::gpu::context::GpuContext;
use crate::gpu::xk_ffi;
use crate::waves::diffraction::{DiffractionRay, PixelPoint};

/// Parameters for wave/screen pixel generation.
#[derive(Debug, Clone)]
pub struct WaveParams {
    /// Screen center position [mm]
    pub center: [f64; 3],
    /// Screen extent in x [mm] (half-width)
    pub dx: f64,
    /// Screen extent in z [mm] (half-height)
    pub dz: f64,
    /// Number of pixels in x
    pub nx: usize,
    /// Number of pixels in z
    pub nz: usize,
}

impl WaveParams {
    pub fn new(center: [f64; 3], dx: f64, dz: f64, nx: usize, nz: usize) -> Self {
        Self { center, dx, dz, nx, nz }
    }

    pub(crate) fn ffi(&self) -> xk_ffi::xk_wave_params {
        xk_ffi::xk_wave_params {
            center: self.center,
            dx: self.dx,
            dz: self.dz,
            nx: self.nx,
            nz: self.nz,
        }
    }
}

fn shared() -> &'static GpuContext {
    GpuContext::shared().expect("no CUDA device")
}

/// Generate a 2D pixel grid for diffraction calculation: nx * nz points,
/// x outer and z inner (z varies fastest).
pub fn prepare_wave(params: &WaveParams) -> Vec<PixelPoint> {
    let m = params.nx * params.nz;
    let (mut x, mut y, mut z) = (vec![0.0; m], vec![0.0; m], vec![0.0; m]);
    if m > 0 {
        let ctx = shared();
        let p = params.ffi();
        let mut out = xk_ffi::xk_pixels_out {
            x: x.as_mut_ptr(),
            y: y.as_mut_ptr(),
            z: z.as_mut_ptr(),
        };
        let rc = unsafe { xk_ffi::xk_prepare_wave(ctx.raw(), &p, &mut out) };
        xk_ffi::check(rc, ctx.raw(), "xk_prepare_wave");
    }
    (0..m).map(|i| PixelPoint { x: x[i], y: y[i], z: z[i] }).collect()
}

/// Host views of the beam columns `beam_to_diffraction_rays` reads; the
/// amplitude columns are split into re/im arrays (the library takes them
/// as separate f64 columns).
pub(crate) struct BeamColumns<'a> {
    beam: &'a Beam,
    amps: Option<[Vec<f64>; 4]>,
}

impl<'a> BeamColumns<'a> {
    pub(crate) fn new(beam: &'a Beam) -> Self {
        let amps = beam.amplitudes().map(|a| {
            let split = |v: &ndarray::Array1<Complex64>, im: bool| {
                v.iter().map(|c| if im { c.im } else { c.re }).collect::<Vec<f64>>()
            };
            [split(&a.es, false), split(&a.es, true), split(&a.ep, false), split(&a.ep, true)]
        });
        Self { beam, amps }
    }

    pub(crate) fn ffi(&self) -> xk_ffi::xk_beam {
        let col = |a: &ndarray::Array1<f64>| {
            a.as_slice().expect("beam columns are contiguous").as_ptr()
        };
        let null = std::ptr::null::<f64>();
        let (er, ei, pr, pi) = match &self.amps {
            Some(a) => (a[0].as_ptr(), a[1].as_ptr(), a[2].as_ptr(), a[3].as_ptr()),
            None => (null, null, null, null),
        };
        xk_ffi::xk_beam {
            x: col(&self.beam.x),
            y: col(&self.beam.y),
            z: col(&self.beam.z),
            a: col(&self.beam.a),
            b: col(&self.beam.b),
            c: col(&self.beam.c),
            e: col(&self.beam.e),
            es_re: er,
            es_im: ei,
            ep_re: pr,
            ep_im: pi,
        }
    }

    pub(crate) fn len(&self) -> usize {
        self.beam.x.len()
    }
}

/// Convert beam data to diffraction rays: ray i is beam ray good[i] with
/// its surface normal, nl = n . (a, b, c), and the beam's amplitudes (1 and
/// 0 without them). Panics on a good index outside the beam, as before.
pub fn beam_to_diffraction_rays(
    beam: &Beam,
    normals: &[[f64; 3]],
    good: &[usize],
) -> Vec<DiffractionRay> {
    let n = good.len();
    let mut c: Vec<Vec<f64>> = (0..12).map(|_| vec![0.0; n]).collect();
    if n > 0 {
        let ctx = shared();
        let cols = BeamColumns::new(beam);
        // A good index must address both a beam ray and a normal; the
        // library rejects larger ones (XK_ERR_INVALID -> panic).
        let n_beam = cols.len().min(normals.len());
        let b = cols.ffi();
        let mut out = xk_ffi::xk_rays_out {
            x: c[0].as_mut_ptr(),
            y: c[1].as_mut_ptr(),
            z: c[2].as_mut_ptr(),
            nx: c[3].as_mut_ptr(),
            ny: c[4].as_mut_ptr(),
            nz: c[5].as_mut_ptr(),
            nl: c[6].as_mut_ptr(),
            es_re: c[7].as_mut_ptr(),
            es_im: c[8].as_mut_ptr(),
            ep_re: c[9].as_mut_ptr(),
            ep_im: c[10].as_mut_ptr(),
            energy: c[11].as_mut_ptr(),
        };
        let rc = unsafe {
            xk_ffi::xk_beam_to_rays(ctx.raw(), &b, n_beam, normals.as_ptr() as *const f64,
                                    good.as_ptr(), n, &mut out)
        };
        xk_ffi::check(rc, ctx.raw(), "xk_beam_to_rays");
    }
    (0..n)
        .map(|i| DiffractionRay {
            x: c[0][i],
            y: c[1][i],
            z: c[2][i],
            nx: c[3][i],
            ny: c[4][i],
            nz: c[5][i],
            nl: c[6][i],
            es: Complex64::new(c[7][i], c[8][i]),
            ep: Complex64::new(c[9][i], c[10][i]),
            energy: c[11][i],
        })
        .collect()
}
