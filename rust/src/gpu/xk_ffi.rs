//! Raw bindings to libxk.so, the sm_100a Kirchhoff engine (C ABI `include/xk.h`).
//!
//! Every struct is `#[repr(C)]` with the field order of its C declaration;
//! every function is the C entry point of the same name. Pointers are host
//! pointers unless a function's documentation in `include/xk.h` says device.
//! The safe wrappers live in `gpu::context`, `gpu::kirchhoff`,
//! `gpu::fallback` and the `waves` modules.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_int, c_void};

// ---- status codes and paths -------------------------------------------------
pub const XK_OK: c_int = 0;
pub const XK_ERR_NO_DEVICE: c_int = 1;
pub const XK_ERR_INVALID: c_int = 2;
pub const XK_ERR_OOM: c_int = 3;
pub const XK_ERR_BUDGET: c_int = 4;
pub const XK_ERR_CUDA: c_int = 5;
pub const XK_ERR_TIMEOUT: c_int = 6;
pub const XK_ERR_NOT_FOUND: c_int = 7;
pub const XK_ERR_CANCELLED: c_int = 8;
pub const XK_ERR_SHUTDOWN: c_int = 9;

pub const XK_PATH_F64: c_int = 0;
pub const XK_PATH_F32PR: c_int = 1;
pub const XK_PATH_SEPARABLE: c_int = 2;
pub const XK_SERVE_SHORTEST_AGED: c_int = 0;
pub const XK_SERVE_EQUAL_SHARE: c_int = 1;

pub const XK_BATCH_DEVICE: c_int = 1;
pub const XK_BATCH_NO_GRAPH: c_int = 2;

pub const XK_NOALLOC_MAX_RAYS: usize = 131072;
pub const XK_NOALLOC_SCRATCH_BYTES: usize = 32 << 20;

// ---- data ---------------------------------------------------------------------

/// Opaque context (one CUDA device, its stream and workspaces).
#[repr(C)]
pub struct xk_ctx {
    _opaque: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_rays {
    pub x: *const f64,
    pub y: *const f64,
    pub z: *const f64,
    pub nx: *const f64,
    pub ny: *const f64,
    pub nz: *const f64,
    pub nl: *const f64,
    pub es_re: *const f64,
    pub es_im: *const f64,
    pub ep_re: *const f64,
    pub ep_im: *const f64,
    pub energy: *const f64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_pixels {
    pub x: *const f64,
    pub y: *const f64,
    pub z: *const f64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_field {
    pub es_re: *mut f64,
    pub es_im: *mut f64,
    pub ep_re: *mut f64,
    pub ep_im: *mut f64,
}

/// Per-call report (`xk_stats`).
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct xk_stats {
    pub pairs: f64,
    pub gpu_ms: f64,
    pub wall_ms: f64,
    pub path: c_int,
    pub kernels: c_int,
    pub n_tiles: c_int,
    pub n_chunks: c_int,
    pub n_items: i64,
    pub phase_bound_rad: f64,
    pub h2d_bytes: f64,
    pub d2h_bytes: f64,
    pub main_kernel_ms: f64,
    pub groups: c_int,
    pub routed_reason: c_int,
    pub sweep: c_int,
    pub one_polarization: c_int,
    pub tuned: c_int,
    pub folded: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct xk_tune_result {
    pub default_ms: f64,
    pub best_ms: f64,
    pub phase_budget: f64,
    pub items_per_warp: i64,
    pub sweep: c_int,
    pub trials: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct xk_pipe_peaks {
    pub fma_lane_ops_per_clk_sm: f64,
    pub mufu_ops_per_clk_sm: f64,
    pub sm_clock_mhz: f64,
    pub fma_ms: f64,
    pub mufu_ms: f64,
    pub num_sms: c_int,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_wave_params {
    pub center: [f64; 3],
    pub dx: f64,
    pub dz: f64,
    pub nx: usize,
    pub nz: usize,
}

/// Beam columns read by `beam_to_diffraction_rays`; the four amplitude
/// pointers are all set or all null.
#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_beam {
    pub x: *const f64,
    pub y: *const f64,
    pub z: *const f64,
    pub a: *const f64,
    pub b: *const f64,
    pub c: *const f64,
    pub e: *const f64,
    pub es_re: *const f64,
    pub es_im: *const f64,
    pub ep_re: *const f64,
    pub ep_im: *const f64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_rays_out {
    pub x: *mut f64,
    pub y: *mut f64,
    pub z: *mut f64,
    pub nx: *mut f64,
    pub ny: *mut f64,
    pub nz: *mut f64,
    pub nl: *mut f64,
    pub es_re: *mut f64,
    pub es_im: *mut f64,
    pub ep_re: *mut f64,
    pub ep_im: *mut f64,
    pub energy: *mut f64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_pixels_out {
    pub x: *mut f64,
    pub y: *mut f64,
    pub z: *mut f64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_fresnel_screen {
    pub x_min: f64,
    pub x_max: f64,
    pub nx: usize,
    pub z_min: f64,
    pub z_max: f64,
    pub nz: usize,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_solve {
    pub rays: xk_rays,
    pub n_rays: usize,
    pub pixels: xk_pixels,
    pub n_pix: usize,
    pub out: xk_field,
}

#[repr(C)]
pub struct xk_batch {
    _opaque: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct xk_batch_stats {
    pub pairs: f64,
    pub plan_ms: f64,
    pub exec_ms: f64,
    pub wall_ms: f64,
    pub n_solves: c_int,
    pub routed_f64: c_int,
    pub kernels: c_int,
    pub graph: c_int,
    pub n_items: i64,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct xk_solve_plan {
    pub path: c_int,
    pub routed_reason: c_int,
    pub n_tiles: c_int,
    pub n_chunks: c_int,
    pub groups: c_int,
    pub sweep: c_int,
    pub phase_bound_rad: f64,
    pub one_polarization: c_int,
    pub tuned: c_int,
}

#[repr(C)]
pub struct xk_server {
    _opaque: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct xk_server_opts {
    pub hbm_budget_bytes: f64,
    pub epoch_pairs: f64,
    pub max_active: c_int,
    pub item_pairs: f64,
    pub inject_alloc_failure_every: c_int,
    pub reserve_sms: c_int,
    pub policy: c_int,
    pub aging_ms: f64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct xk_request {
    pub rays: xk_rays,
    pub n_rays: usize,
    pub rayset: u64,
    pub pixels: xk_pixels,
    pub n_pix: usize,
    pub out: xk_field,
    pub path: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct xk_request_stats {
    pub pairs: f64,
    pub queue_ms: f64,
    pub plan_ms: f64,
    pub run_ms: f64,
    pub total_ms: f64,
    pub path: c_int,
    pub epochs: c_int,
    pub status: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct xk_server_stats {
    pub submitted: i64,
    pub completed: i64,
    pub failed: i64,
    pub epochs: i64,
    pub kernels: i64,
    pub pending: i64,
    pub active: i64,
    pub pairs_done: f64,
    pub used_bytes: f64,
    pub peak_bytes: f64,
    pub resident_ray_bytes: f64,
    pub pairs_launched: f64,
}

// `xk_gpu_ray` / `xk_gpu_pixel` are `gpu::kirchhoff::GpuRay` / `GpuPixel`
// themselves (same #[repr(C)] field order, 48 and 16 bytes).
use crate::gpu::kirchhoff::{GpuPixel, GpuRay};

#[link(name = "xk")]
unsafe extern "C" {
    // context and diagnostics
    pub fn xk_init(device: c_int, out: *mut *mut xk_ctx) -> c_int;
    pub fn xk_shared(out: *mut *mut xk_ctx) -> c_int;
    pub fn xk_destroy(ctx: *mut xk_ctx);
    pub fn xk_device_name(ctx: *const xk_ctx) -> *const c_char;
    pub fn xk_last_error(ctx: *const xk_ctx) -> *const c_char;
    pub fn xk_status_string(status: c_int) -> *const c_char;
    pub fn xk_version() -> *const c_char;
    pub fn xk_route_reason(reason: c_int) -> *const c_char;
    pub fn xk_set_option(ctx: *mut xk_ctx, name: *const c_char, value: f64) -> c_int;
    pub fn xk_autotune(ctx: *mut xk_ctx, rays: *const xk_rays, n_rays: usize,
                       pixels: *const xk_pixels, n_pix: usize, out: *mut xk_field,
                       budget_ms: f64, apply: c_int, result: *mut xk_tune_result) -> c_int;

    pub fn xk_probe_pipes(ctx: *mut xk_ctx, out: *mut xk_pipe_peaks) -> c_int;

    // single solves
    pub fn xk_diffraction_integral(ctx: *mut xk_ctx, rays: *const xk_rays, n_rays: usize,
                                   pixels: *const xk_pixels, n_pix: usize, out: *mut xk_field,
                                   path: c_int, stats: *mut xk_stats) -> c_int;
    pub fn xk_diffraction_integral_device(ctx: *mut xk_ctx, rays: *const xk_rays, n_rays: usize,
                                          pixels: *const xk_pixels, n_pix: usize,
                                          out: *mut xk_field, path: c_int, stream: *mut c_void,
                                          stats: *mut xk_stats) -> c_int;
    pub fn xk_kirchhoff_gpu(ctx: *mut xk_ctx, rays: *const GpuRay, n_rays: usize,
                            pixels: *const GpuPixel, n_pix: usize, out: *mut f64) -> c_int;
    pub fn xk_kirchhoff_auto(rays: *const GpuRay, n_rays: usize, pixels: *const GpuPixel,
                             n_pix: usize, out: *mut f64) -> c_int;

    // producers and the chained beam solve
    pub fn xk_prepare_wave(ctx: *mut xk_ctx, params: *const xk_wave_params,
                           out: *mut xk_pixels_out) -> c_int;
    pub fn xk_beam_to_rays(ctx: *mut xk_ctx, beam: *const xk_beam, n_beam: usize,
                           normals: *const f64, good: *const usize, n_good: usize,
                           out: *mut xk_rays_out) -> c_int;
    pub fn xk_diffraction_beam(ctx: *mut xk_ctx, beam: *const xk_beam, n_beam: usize,
                               normals: *const f64, good: *const usize, n_good: usize,
                               params: *const xk_wave_params, out: *mut xk_field, path: c_int,
                               stats: *mut xk_stats) -> c_int;

    // 2-D Fresnel
    pub fn xk_fresnel_propagate(ctx: *mut xk_ctx, ray_x: *const f64, ray_z: *const f64,
                                es_re: *const f64, es_im: *const f64, n_rays: usize,
                                energy: f64, dist: f64, screen: *const xk_fresnel_screen,
                                amp_re: *mut f64, amp_im: *mut f64, x_pixels: *mut f64,
                                z_pixels: *mut f64, path: c_int, stats: *mut xk_stats) -> c_int;

    // batches
    pub fn xk_batch_create(ctx: *mut xk_ctx, solves: *const xk_solve, n: usize, path: c_int,
                           flags: c_int, out: *mut *mut xk_batch) -> c_int;
    pub fn xk_batch_run(batch: *mut xk_batch, stats: *mut xk_batch_stats) -> c_int;
    pub fn xk_batch_solve_plan(batch: *const xk_batch, i: usize, out: *mut xk_solve_plan) -> c_int;
    pub fn xk_batch_destroy(batch: *mut xk_batch);

    // serving
    pub fn xk_server_create(ctx: *mut xk_ctx, opts: *const xk_server_opts,
                            out: *mut *mut xk_server) -> c_int;
    pub fn xk_server_upload_rays(server: *mut xk_server, rays: *const xk_rays, n: usize,
                                 handle: *mut u64) -> c_int;
    pub fn xk_server_release_rays(server: *mut xk_server, handle: u64) -> c_int;
    pub fn xk_server_upload_beam(server: *mut xk_server, beam: *const xk_beam, n_beam: usize,
                                 normals: *const f64, good: *const usize, n_good: usize,
                                 handle: *mut u64) -> c_int;
    pub fn xk_server_submit(server: *mut xk_server, req: *const xk_request,
                            ticket: *mut u64) -> c_int;
    pub fn xk_server_wait(server: *mut xk_server, ticket: u64, timeout_ms: f64,
                          stats: *mut xk_request_stats) -> c_int;
    pub fn xk_server_get_stats(server: *mut xk_server, out: *mut xk_server_stats) -> c_int;
    pub fn xk_server_destroy(server: *mut xk_server);

    // allocation-free FP64 solve (device pointers; stream is a cudaStream_t or null)
    pub fn xk_diffraction_f64_noalloc(rays: *const xk_rays, n_rays: usize,
                                      pixels: *const xk_pixels, n_pix: usize,
                                      out: *mut xk_field, stream: *mut c_void) -> c_int;
}

/// Panics with the library's message for a non-zero status, as the reference
/// panics on a failed GPU readback (src/gpu/kirchhoff.rs:268-271).
pub fn check(status: c_int, ctx: *const xk_ctx, what: &str) {
    if status == XK_OK {
        return;
    }
    let text = |p: *const c_char| {
        if p.is_null() {
            String::new()
        } else {
            unsafe { std::ffi::CStr::from_ptr(p) }.to_string_lossy().into_owned()
        }
    };
    let code = text(unsafe { xk_status_string(status) });
    let detail = if ctx.is_null() { String::new() } else { text(unsafe { xk_last_error(ctx) }) };
    panic!("{what} failed: {code} ({status}) {detail}");
}
