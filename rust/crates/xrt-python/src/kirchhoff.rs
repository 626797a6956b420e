//! PyO3 binding of the Kirchhoff integral on the sm_100a engine.
//!
//! `diffraction_integral_rs` keeps its name, its 15 list arguments, its
//! ValueError on mismatched lengths and its 4-list result; the columns go to
//! libxk.so as they arrive (structure of arrays), without building
//! `DiffractionRay` records. Register it in the module as before:
//! `m.add_function(wrap_pyfunction!(kirchhoff::diffraction_integral_rs, m)?)?`.

use pyo3::prelude::*;

use xrt_rs::gpu::context::GpuContext;
use xrt_rs::gpu::xk_ffi;

fn check_equal_lengths(pairs: &[(&str, usize)]) -> PyResult<()> {
    if let Some(&(first, n)) = pairs.first() {
        for &(name, len) in &pairs[1..] {
            if len != n {
                return Err(pyo3::exceptions::PyValueError::new_err(format!(
                    "array length mismatch: {name} has {len} elements but {first} has {n}"
                )));
            }
        }
    }
    Ok(())
}

/// Kirchhoff diffraction integral, FP64 path on the GPU.
///
/// Args: ray positions, normals, obliquity, s- and p-amplitudes (re, im),
/// energies [eV]; pixel positions [mm].
/// Returns: (es_re, es_im, ep_re, ep_im) at the pixels.
#[pyfunction]
#[allow(clippy::too_many_arguments)]
pub fn diffraction_integral_rs(
    ray_x: Vec<f64>,
    ray_y: Vec<f64>,
    ray_z: Vec<f64>,
    ray_nx: Vec<f64>,
    ray_ny: Vec<f64>,
    ray_nz: Vec<f64>,
    ray_nl: Vec<f64>,
    ray_es_re: Vec<f64>,
    ray_es_im: Vec<f64>,
    ray_ep_re: Vec<f64>,
    ray_ep_im: Vec<f64>,
    ray_energy: Vec<f64>,
    pix_x: Vec<f64>,
    pix_y: Vec<f64>,
    pix_z: Vec<f64>,
) -> PyResult<(Vec<f64>, Vec<f64>, Vec<f64>, Vec<f64>)> {
    let n = ray_x.len();
    check_equal_lengths(&[
        ("ray_x", n),
        ("ray_y", ray_y.len()),
        ("ray_z", ray_z.len()),
        ("ray_nx", ray_nx.len()),
        ("ray_ny", ray_ny.len()),
        ("ray_nz", ray_nz.len()),
        ("ray_nl", ray_nl.len()),
        ("ray_es_re", ray_es_re.len()),
        ("ray_es_im", ray_es_im.len()),
        ("ray_ep_re", ray_ep_re.len()),
        ("ray_ep_im", ray_ep_im.len()),
        ("ray_energy", ray_energy.len()),
    ])?;
    check_equal_lengths(&[("pix_x", pix_x.len()), ("pix_y", pix_y.len()), ("pix_z", pix_z.len())])?;
    let m = pix_x.len();
    let (mut es_re, mut es_im, mut ep_re, mut ep_im) =
        (vec![0.0; m], vec![0.0; m], vec![0.0; m], vec![0.0; m]);
    if m == 0 {
        return Ok((es_re, es_im, ep_re, ep_im));
    }
    let ctx = GpuContext::shared()
        .ok_or_else(|| pyo3::exceptions::PyRuntimeError::new_err("no CUDA device"))?;
    let rays = xk_ffi::xk_rays {
        x: ray_x.as_ptr(),
        y: ray_y.as_ptr(),
        z: ray_z.as_ptr(),
        nx: ray_nx.as_ptr(),
        ny: ray_ny.as_ptr(),
        nz: ray_nz.as_ptr(),
        nl: ray_nl.as_ptr(),
        es_re: ray_es_re.as_ptr(),
        es_im: ray_es_im.as_ptr(),
        ep_re: ray_ep_re.as_ptr(),
        ep_im: ray_ep_im.as_ptr(),
        energy: ray_energy.as_ptr(),
    };
    let pix = xk_ffi::xk_pixels { x: pix_x.as_ptr(), y: pix_y.as_ptr(), z: pix_z.as_ptr() };
    let mut out = xk_ffi::xk_field {
        es_re: es_re.as_mut_ptr(),
        es_im: es_im.as_mut_ptr(),
        ep_re: ep_re.as_mut_ptr(),
        ep_im: ep_im.as_mut_ptr(),
    };
    let rc = unsafe {
        xk_ffi::xk_diffraction_integral(ctx.raw(), &rays, n, &pix, m, &mut out,
                                        xk_ffi::XK_PATH_F64, std::ptr::null_mut())
    };
    if rc != xk_ffi::XK_OK {
        return Err(pyo3::exceptions::PyRuntimeError::new_err(format!(
            "xk_diffraction_integral failed with status {rc}"
        )));
    }
    Ok((es_re, es_im, ep_re, ep_im))
}
