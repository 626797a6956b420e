//! GPU context: one CUDA device of the sm_100a Kirchhoff engine (libxk.so).
//!
//! Same public surface as before (`new`, `shared`, `adapter_name`); the
//! handle owns the device's stream and workspaces inside the library instead
//! of a wgpu device and queue. Calls on one context are serialised inside the
//! library, so the shared context can be used from many threads (Rayon).

use std::ffi::CStr;
use std::sync::OnceLock;

use crate::gpu::xk_ffi;

/// GPU context holding a libxk device context.
pub struct GpuContext {
    pub(crate) handle: *mut xk_ffi::xk_ctx,
    owned: bool,
}

// The library guards each context with its own mutex.
unsafe impl Send for GpuContext {}
unsafe impl Sync for GpuContext {}

impl GpuContext {
    /// A private context on CUDA device 0. Returns None if there is no
    /// usable device.
    pub fn new() -> Option<Self> {
        let mut h = std::ptr::null_mut();
        let rc = unsafe { xk_ffi::xk_init(0, &mut h) };
        (rc == xk_ffi::XK_OK && !h.is_null()).then_some(Self { handle: h, owned: true })
    }

    /// The process-wide context, created at most once (None without a device).
    pub fn shared() -> Option<&'static Self> {
        static SHARED: OnceLock<Option<GpuContext>> = OnceLock::new();
        SHARED
            .get_or_init(|| {
                let mut h = std::ptr::null_mut();
                let rc = unsafe { xk_ffi::xk_shared(&mut h) };
                (rc == xk_ffi::XK_OK && !h.is_null()).then_some(Self { handle: h, owned: false })
            })
            .as_ref()
    }

    /// Name of the CUDA device.
    pub fn adapter_name(&self) -> &str {
        let p = unsafe { xk_ffi::xk_device_name(self.handle) };
        if p.is_null() {
            return "";
        }
        unsafe { CStr::from_ptr(p) }.to_str().unwrap_or("")
    }

    /// Sets one of the library's tuning options ("phase_budget", "sweep", ...).
    pub fn set_option(&self, name: &str, value: f64) {
        let c = std::ffi::CString::new(name).expect("option name without NUL");
        let rc = unsafe { xk_ffi::xk_set_option(self.handle, c.as_ptr(), value) };
        xk_ffi::check(rc, self.handle, "xk_set_option");
    }

    /// The library handle, for direct `xk_ffi` calls (valid while `self` lives).
    pub fn raw(&self) -> *mut xk_ffi::xk_ctx {
        self.handle
    }
}

impl Drop for GpuContext {
    fn drop(&mut self) {
        // The shared context lives for the whole process.
        if self.owned {
            unsafe { xk_ffi::xk_destroy(self.handle) }
        }
    }
}

impl std::fmt::Debug for GpuContext {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        f.debug_struct("GpuContext").field("device", &self.adapter_name()).finish()
    }
}
