// Internal declarations shared by the xk CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "../../include/xk.h"

namespace xk {

// c*hbar [eV*Angstrom], src/core/consts.rs:74; k = E / CHBAR * 1e7 [1/mm].
constexpr double kChbar = 1973.2697177417986;
constexpr double kPi = 3.14159265358979323846;

// Status carrying a message; the API layer copies it into the context.
struct Status {
    int code = XK_OK;
    std::string msg;
    bool ok() const { return code == XK_OK; }
    static Status Ok() { return Status{}; }
    static Status Err(int c, std::string m) { return Status{c, std::move(m)}; }
    static Status FromCuda(cudaError_t e) {
        return e == cudaSuccess ? Ok() : Err(XK_ERR_CUDA, cudaGetErrorString(e));
    }
};

#define XK_CUDA_TRY(expr)                                                                  \
    do {                                                                                   \
        cudaError_t err__ = (expr);                                                        \
        if (err__ != cudaSuccess) {                                                        \
            return ::xk::Status::Err(err__ == cudaErrorMemoryAllocation ? XK_ERR_OOM       \
                                                                        : XK_ERR_CUDA,     \
                                     std::string(#expr) + ": " + cudaGetErrorString(err__)); \
        }                                                                                  \
    } while (0)

#define XK_TRY(expr)                      \
    do {                                  \
        ::xk::Status st__ = (expr);       \
        if (!st__.ok()) return st__;      \
    } while (0)

// NVTX range for the enclosing scope (header-only NVTX v3: a no-op unless a
// profiler is attached), so that planning, epochs and copies show up as
// named ranges on a timeline.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Keeps memory freed to the device's default stream-ordered pool in the pool
// (instead of returning it to the driver at every synchronisation), so that
// repeated batch and server allocations of similar sizes are reused.
inline Status keep_pool_memory(int device) {
    cudaMemPool_t pool;
    XK_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t threshold = UINT64_MAX;
    XK_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    return Status::Ok();
}

// A growable device buffer (never shrinks until freed). With `async_stream`
// set it allocates and frees stream-ordered (cudaMallocAsync/cudaFreeAsync on
// that stream), which never waits for other streams' work.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t async_stream = nullptr;
    Status ensure(size_t want) {
        if (want <= bytes) return Status::Ok();
        release();
        size_t rounded = (want + ((size_t)1 << 20) - 1) & ~(((size_t)1 << 20) - 1);
        if (async_stream) {
            XK_CUDA_TRY(cudaMallocAsync(&ptr, rounded, async_stream));
        } else {
            XK_CUDA_TRY(cudaMalloc(&ptr, rounded));
        }
        bytes = rounded;
        return Status::Ok();
    }
    void release() {
        if (ptr) {
            if (async_stream) cudaFreeAsync(ptr, async_stream);
            else cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};

// Device-pointer views used by the launchers.
struct RaysDev {
    const double *x, *y, *z, *nx, *ny, *nz, *nl, *es_re, *es_im, *ep_re, *ep_im, *energy;
};
struct PixDev {
    const double *x, *y, *z;
};
struct FieldDev {
    double *es_re, *es_im, *ep_re, *ep_im;
};

// Scratch owned by a context for the FP64 plain path.
struct F64Workspace {
    DevBuf rays;      // packed ray records
    DevBuf partials;  // split-ray partial sums
    // false: sin/cos of each phase k|p - r| by the library functions, as the
    // reference computes them; true: an FMA-based reduction by 2 pi first
    // (same phase, same parity bar, about twice as fast at 1e10-1e13 rad).
    bool fast_reduction = false;
};

struct LaunchReport {
    int kernels = 0;
    float gpu_ms = 0.f;
};

// Ray-range splits of the FP64 path for a solve (and the rays per range).
size_t f64_splits(size_t n_rays, size_t n_pix, int num_sms, size_t* rays_per_split);

// Grows `ws` to what f64_enqueue needs for this solve, so a later enqueue
// allocates nothing (e.g. while a CUDA graph is being captured).
Status f64_reserve(size_t n_rays, size_t n_pix, int num_sms, F64Workspace& ws);

// FP64 plain path (xk_f64.cu). All pointers are device pointers; the call
// enqueues on `stream` and does not synchronise.
Status f64_enqueue(const RaysDev& rays, size_t n_rays, const PixDev& pix, size_t n_pix,
                   const FieldDev& out, F64Workspace& ws, cudaStream_t stream, int num_sms,
                   LaunchReport* rep);

// Screen grid and beam-to-ray producers (xk_wave.cu), enqueued on `stream`.
struct WaveGrid {
    double cx, cy, cz, dx, dz;
    size_t nx, nz;
};
struct BeamDev {
    const double *x, *y, *z, *a, *b, *c, *e, *es_re, *es_im, *ep_re, *ep_im;  // amplitudes may be null
    const double* normals;  // n_beam rows of 3
};
// Writes nx*nz points into x/y/z (device arrays).
Status wave_enqueue(const WaveGrid& g, double* x, double* y, double* z, cudaStream_t stream);
// Gathers the rays of `good` (device array of n_good indices < n_beam) into
// the 12 device columns of `out` (x, y, z, nx, ny, nz, nl, es_re, es_im,
// ep_re, ep_im, energy).
Status beam_rays_enqueue(const BeamDev& beam, const uint64_t* good, size_t n_good,
                         double* const out[12], cudaStream_t stream);

// ---- 2-D Fresnel propagation (xk_fresnel.cu) ------------------------------

struct FresnelIn {
    const double *rx, *rz, *er, *ei;  // device, n each
    size_t n;
    double energy, dist;
    double x_min, x_max, z_min, z_max;
    size_t nx, nz;
    double max_amp;                   // max_j |es_j| (scales the f16 factors)
    double max_rx_off, max_rz_off;    // max_j |x_j - screen centre x|, same for z
    double *out_re, *out_im;          // device, nx * nz each
    bool finite = true;               // every ray coordinate and amplitude is finite
};

struct FresnelShape {
    size_t m_pad = 0, n_pad = 0;  // padded rows of A (screen z) and B (2 x screen x)
    size_t tiles = 0;             // 128 x 256 output tiles (one per CTA)
    bool pair = false;            // CTA pairs (256 x 256 tiles, one MMA over two SMs)
    int ray_blocks = 0;           // blocks of 32 rays (the contraction)
    int splits = 1;               // K splits per output tile
};

struct FresnelWorkspace {
    DevBuf coords, partial, ctrl;
    uint32_t wait_limit = 1u << 24;  // polls of every bounded wait of the tensor-core product
    bool allow_pair = true;          // CTA-pair product on screens of more than 128 rows
    uint32_t stall_once = 0;         // test hook: the next product's first stage never completes
};

struct FresnelReport {
    int kernels = 0;
    double gemm_ms = 0.0;                       // device time of the tensor-core products
    cudaEvent_t ev_gemm[2] = {nullptr, nullptr};  // set to time the products (synchronises per chunk)
    FresnelShape shape;
    int* d_err = nullptr;                       // device error word of the products
    int used_path = 0;                          // XK_PATH_* that ran
};

FresnelShape fresnel_shape(size_t n, size_t nx, size_t nz, int num_sms, bool allow_pair = true);

// Enqueues screen coordinates into ws.coords (nx then nz doubles; the caller
// sizes it) and the sum for `path` (XK_PATH_F64 or XK_PATH_SEPARABLE).
Status fresnel_enqueue(const FresnelIn& in, FresnelWorkspace& ws, cudaStream_t stream,
                       int num_sms, int path, FresnelReport* rep);

// GpuRay / GpuPixel records (f32 AoS, src/gpu/kirchhoff.rs:20-45) on the
// device -> the f64 SoA columns the solvers read (exact widening), and the
// solved field -> 4 doubles per pixel, the layout of Vec<(Complex64,
// Complex64)> (xk_wave.cu).
Status gpu_records_enqueue(const xk_gpu_ray* rays, size_t n, const xk_gpu_pixel* pix, size_t m,
                           double* const ray_cols[12], double* px, double* py, double* pz,
                           cudaStream_t stream);
Status interleave_field_enqueue(const FieldDev& f, size_t m, double* out, cudaStream_t stream);

}  // namespace xk
