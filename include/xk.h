/*
 * xk — B200-native Kirchhoff diffraction engine, C ABI.
 *
 * Drop-in boundary for the Kirchhoff path of physwkim/xrt-rs. Every entry
 * point takes plain pointers and sizes; nothing in these signatures is a
 * torch or CUDA-runtime type (streams are passed as `void*`, i.e. a
 * cudaStream_t or NULL for the library's own stream).
 *
 * Units and conventions follow the reference: positions in mm, energies in
 * eV, k = E / CHBAR * 1e7 mm^-1 with CHBAR = 1973.2697177417986 eV*A
 * (src/core/consts.rs:74). For every screen point p the library returns
 *   Es(p) = sum_j es_j * U_j(p),  Ep(p) = sum_j ep_j * U_j(p),
 *   U_j(p) = i*k_j/(4*pi) * (nl_j + n_j.(p - r_j)/|p - r_j|) * exp(i*k_j*|p - r_j|) / |p - r_j|,
 * skipping rays with |p - r_j| < 1e-30 (src/waves/diffraction.rs:67-117).
 *
 * Two compute paths:
 *   XK_PATH_F64    the reference algorithm run directly in FP64 on the GPU,
 *                  per-pixel complex Kahan summation (the parity path).
 *   XK_PATH_F32PR  FP32 phase-reduced form: per (screen tile, ray chunk)
 *                  item the phase is split into FP64 per-pixel and per-ray
 *                  parts and an FP32 residual, compensated two-float
 *                  accumulation, FP64 cross-chunk reduction. Solves it cannot
 *                  bound (mixed energies within a chunk, rays touching the
 *                  screen) are routed to XK_PATH_F64 and reported in stats.
 *
 * Every call blocks until its results are in the caller's buffers, like the
 * reference's pollster::block_on (src/gpu/kirchhoff.rs:82). Calls on one
 * context are serialised by a mutex; use one context per thread for
 * concurrency, or the server API for continuous batching.
 *
 * There is no CPU fallback: without a CUDA device every compute entry point
 * returns XK_ERR_NO_DEVICE.
 */
#ifndef XK_H
#define XK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
    XK_OK = 0,
    XK_ERR_NO_DEVICE = 1, /* no usable CUDA device */
    XK_ERR_INVALID = 2,   /* null pointer, length mismatch, size out of range */
    XK_ERR_OOM = 3,       /* device or pinned-host allocation failed */
    XK_ERR_BUDGET = 4,    /* request larger than the configured HBM budget */
    XK_ERR_CUDA = 5,      /* CUDA runtime or kernel error */
    XK_ERR_TIMEOUT = 6,   /* a bounded wait ran out */
    XK_ERR_NOT_FOUND = 7, /* unknown handle or ticket */
    XK_ERR_CANCELLED = 8, /* request cancelled before completion */
    XK_ERR_SHUTDOWN = 9   /* server is shutting down */
};

enum { XK_PATH_F64 = 0, XK_PATH_F32PR = 1, XK_PATH_SEPARABLE = 2 };

/* ---- data structures --------------------------------------------------- */

/* Rays on the optical element, structure of arrays, one f64 per ray in each
 * array. Field meaning follows DiffractionRay (src/waves/diffraction.rs:16-33)
 * and the argument order of diffraction_integral_rs
 * (crates/xrt-python/src/lib.rs:323-339). */
typedef struct xk_rays {
    const double *x, *y, *z;     /* position [mm] */
    const double *nx, *ny, *nz;  /* surface normal */
    const double *nl;            /* obliquity factor n.l */
    const double *es_re, *es_im; /* s-polarised amplitude */
    const double *ep_re, *ep_im; /* p-polarised amplitude */
    const double *energy;        /* [eV] */
} xk_rays;

/* Screen points (PixelPoint, src/waves/diffraction.rs:36-41). */
typedef struct xk_pixels {
    const double *x, *y, *z;
} xk_pixels;

/* Output field per screen point (DiffractionResult, diffraction.rs:44-48). */
typedef struct xk_field {
    double *es_re, *es_im, *ep_re, *ep_im;
} xk_field;

/* GpuRay, 48 bytes, f32 (src/gpu/kirchhoff.rs:20-35). */
typedef struct xk_gpu_ray {
    float x, y, z, nx, ny, nz, nl, energy, es_re, es_im, ep_re, ep_im;
} xk_gpu_ray;

/* GpuPixel, 16 bytes (src/gpu/kirchhoff.rs:38-45). */
typedef struct xk_gpu_pixel {
    float x, y, z, _pad;
} xk_gpu_pixel;

/* Per-call report. */
typedef struct xk_stats {
    double pairs;            /* n_rays * n_pix */
    double gpu_ms;           /* device time of the compute kernels (CUDA events) */
    double wall_ms;          /* host wall time of the whole call incl. copies */
    int path;                /* XK_PATH_* actually used */
    int kernels;             /* kernel launches issued by the call */
    int n_tiles;             /* screen tiles (F32PR) */
    int n_chunks;            /* ray chunks (F32PR) */
    long long n_items;       /* work items (F32PR) */
    double phase_bound_rad;  /* planner's bound on the FP32 residual phase */
    double h2d_bytes, d2h_bytes;
    double main_kernel_ms;   /* device time of the pair kernel alone (CUDA events) */
    int groups;              /* ray groups per tile (F32PR) */
    int routed_reason;       /* 0 = not routed; see xk_route_reason() */
    int sweep;               /* F32PR sweep used: 0 SFU reciprocal, 1 packed + quadratic series,
                                2 packed + linear series; XK_PATH_SEPARABLE (Fresnel): 1 CTA-pair
                                tiles, 0 one CTA per tile; -1 none */
    int one_polarization;    /* F32PR: 1 if every ray had ray 0's polarization, so the kernel
                                summed one amplitude column and Ep = (ep_0 / es_0) Es */
    int tuned;               /* F32PR: 1 if the solve used autotuned settings of its bucket */
    int folded;              /* F32PR: 1 if the kernel folded each point's base phase into the
                                per-pair phase (near field) */
} xk_stats;

/* ---- context ------------------------------------------------------------ */
typedef struct xk_ctx xk_ctx;

/* GpuContext::new (src/gpu/context.rs:20-22,33-67): create a context on CUDA
 * device `device`. Returns XK_ERR_NO_DEVICE when there is none. */
int xk_init(int device, xk_ctx** out);

/* GpuContext::shared (src/gpu/context.rs:28-31): the process-wide context on
 * device 0, created at most once. *out is NULL when no device exists. */
int xk_shared(xk_ctx** out);

/* Frees a context made by xk_init (the shared one is never freed). */
void xk_destroy(xk_ctx* ctx);

/* GpuContext::adapter_name (src/gpu/context.rs:70-72). */
const char* xk_device_name(const xk_ctx* ctx);

/* Message of the last failure on this context ("" if none). */
const char* xk_last_error(const xk_ctx* ctx);

/* Static description of a status code. */
const char* xk_status_string(int status);

/* Library version string. */
const char* xk_version(void);

/* Why an XK_PATH_F32PR request ran on XK_PATH_F64 (xk_stats.routed_reason). */
const char* xk_route_reason(int reason);

/* Tuning knobs of the F32PR path (no counterpart in the reference, whose
 * shader has no parameters). Names:
 *   "phase_budget"   cap on the FP32 residual phase in rad (default 512)
 *   "tolerance"      requested relative L2 error of the phase-reduced field
 *                    (default 1e-4, range [1e-7, 1e-2]); the residual-phase
 *                    budget is derived from it (and capped by "phase_budget")
 *   "sweep"          -1 automatic, 0 SFU reciprocal, 1 packed f32x2 sweep with
 *                    the quadratic series reciprocal, 2 packed with the linear
 *                    series (automatic where its error stays below a tenth of
 *                    the tolerance)
 *   "groups"         ray ranges per screen tile, 0 = automatic
 *   "items_per_warp" target work items per resident warp (automatic groups)
 *   "polarization"   -1 (default): when every ray's (es, ep) is a multiple of
 *                    ray 0's (to 2^-24), sum one amplitude column and scale it
 *                    for Es and Ep; 0: always sum Es and Ep separately
 *   "f64_reduction"  XK_PATH_F64 only: 0 (default) evaluates sin/cos of each
 *                    FP64 phase with the library functions, as the reference
 *                    does; 1 first reduces the phase by 2 pi with an FMA-based
 *                    Cody-Waite step (same phase value and 1e-10 parity, about
 *                    twice the throughput at phases of 1e10-1e13 rad)
 *   "wait_limit"     polls of every bounded device-side wait (mbarrier waits of
 *                    the phase-reduced kernel and of the tensor-core Fresnel
 *                    product) before the kernel gives up and the call returns
 *                    XK_ERR_TIMEOUT; 1..2^31, default 2^24
 *   "inject_stall"   test hook: the next phase-reduced execution on this
 *                    context arms its first ray stage's barrier with this many
 *                    bytes (a positive multiple of 16, at most 1024) beyond its
 *                    copy, so that stage can never complete and the bounded
 *                    wait runs out; cleared after that one execution
 *   "fresnel_stall"  test hook: 1 makes the next tensor-core Fresnel product on
 *                    this context arm its first stage's barrier with one
 *                    arrival more than its producers make, so the MMA issuer's
 *                    bounded wait runs out (XK_ERR_TIMEOUT); no MMA is issued
 *                    and nothing stays in flight; cleared after that execution
 *   "fresnel_pair"   XK_PATH_SEPARABLE: 1 (default) computes screens of more
 *                    than 128 rows on CTA pairs (one tcgen05 MMA over two SMs,
 *                    256 x 256 tiles); 0 keeps one CTA per 128 x 256 tile */
int xk_set_option(xk_ctx* ctx, const char* name, double value);

typedef struct xk_tune_result {
    double default_ms;       /* device time of the solve with the options in force */
    double best_ms;          /* device time with the best options found */
    double phase_budget;     /* best "phase_budget" (ray-chunk size) */
    long long items_per_warp;/* best "items_per_warp" (ray groups per tile) */
    int sweep;               /* best "sweep" */
    int trials;
} xk_tune_result;

/* Autotuner (no counterpart in the reference): times the XK_PATH_F32PR solve
 * of this device-resident problem under candidate settings of the knobs above
 * (residual-phase budget, i.e. ray-chunk size, never above what the
 * tolerance allows; work items per warp, i.e. ray groups per tile; sweep
 * variant) until `budget_ms` of device time is spent, and writes the field
 * into `out`. With `apply` the fastest settings are kept in the context's
 * tuning cache for this problem's bucket — energy and ray/screen distance to
 * the nearest power of two, ray and screen-point counts by their leading
 * power of two — and every later F32PR solve of that bucket on the context
 * (single calls, batches, servers created afterwards) uses them
 * (xk_stats.tuned); the context's defaults do not change. Options
 * "use_tuned" (1 default, 0 ignores the cache) and "clear_tuned" (any value)
 * control the cache. */
int xk_autotune(xk_ctx* ctx, const xk_rays* rays, size_t n_rays, const xk_pixels* pixels,
                size_t n_pix, xk_field* out, double budget_ms, int apply,
                xk_tune_result* result);

/* Peak rates of the two pipes the phase-reduced pair kernel is bound by (no
 * counterpart in the reference; a measurement aid for rooflines). */
typedef struct xk_pipe_peaks {
    double fma_lane_ops_per_clk_sm; /* FP32 FMA-pipe lane operations per SM clock
                                       (an f32x2 FMA counts two) */
    double mufu_ops_per_clk_sm;     /* sin/cos results of the MUFU unit per SM clock */
    double sm_clock_mhz;            /* SM clock seen during the probe */
    double fma_ms, mufu_ms;         /* device time of each probe */
    int num_sms;
} xk_pipe_peaks;

/* Measures both rates with every SM busy (clock64 cycle counts of resident
 * blocks, so the rates do not depend on the clock). Takes ~0.1 s. */
int xk_probe_pipes(xk_ctx* ctx, xk_pipe_peaks* out);

/* ---- single solves --------------------------------------------------------- */

/* waves::diffraction::diffraction_integral (src/waves/diffraction.rs:56-64)
 * and the PyO3 wrapper diffraction_integral_rs
 * (crates/xrt-python/src/lib.rs:321-393). Host buffers in, host buffers out.
 * `path` is XK_PATH_F64 (parity with the reference) or XK_PATH_F32PR.
 * n_rays == 0 yields zeros; n_pix == 0 is a no-op. `stats` may be NULL. */
int xk_diffraction_integral(xk_ctx* ctx, const xk_rays* rays, size_t n_rays,
                            const xk_pixels* pixels, size_t n_pix, xk_field* out,
                            int path, xk_stats* stats);

/* Same with every pointer in rays/pixels/out a DEVICE pointer, launched on
 * `stream` (cudaStream_t, NULL = the context's stream). Returns after the
 * results are written and the stream is synchronised. */
int xk_diffraction_integral_device(xk_ctx* ctx, const xk_rays* rays, size_t n_rays,
                                   const xk_pixels* pixels, size_t n_pix, xk_field* out,
                                   int path, void* stream, xk_stats* stats);

/* gpu::kirchhoff::kirchhoff_gpu (src/gpu/kirchhoff.rs:77-83): GpuRay /
 * GpuPixel records in, (Es, Ep) per pixel out as 4 doubles per pixel
 * (es.re, es.im, ep.re, ep.im) — the memory layout of
 * Vec<(Complex64, Complex64)>. Runs XK_PATH_F32PR with the base phase
 * restored in FP64. */
int xk_kirchhoff_gpu(xk_ctx* ctx, const xk_gpu_ray* rays, size_t n_rays,
                     const xk_gpu_pixel* pixels, size_t n_pix, double* out);

/* gpu::fallback::kirchhoff_auto (src/gpu/fallback.rs:19-26) on the shared
 * context. Unlike the reference there is no CPU fallback: with no device it
 * returns XK_ERR_NO_DEVICE. */
int xk_kirchhoff_auto(const xk_gpu_ray* rays, size_t n_rays, const xk_gpu_pixel* pixels,
                      size_t n_pix, double* out);

/* ---- screens and rays from a beam -----------------------------------------
 *
 * The two producers in front of the path (src/waves/prepare_wave.rs), run on
 * the device so that a beam's columns go to the GPU once and neither the
 * screen grid nor the ray records make a host round trip. */

/* WaveParams (src/waves/prepare_wave.rs:11-23). */
typedef struct xk_wave_params {
    double center[3]; /* screen centre [mm] */
    double dx, dz;    /* half-widths in x and z [mm] */
    size_t nx, nz;    /* points along x and along z */
} xk_wave_params;

/* The columns of core::beam::Beam that beam_to_diffraction_rays reads, one
 * f64 per beam ray in each array. The four amplitude arrays are either all
 * set or all NULL (a beam without amplitudes: es = 1, ep = 0). */
typedef struct xk_beam {
    const double *x, *y, *z;  /* position [mm] */
    const double *a, *b, *c;  /* direction cosines */
    const double *e;          /* energy [eV] */
    const double *es_re, *es_im, *ep_re, *ep_im;
} xk_beam;

/* Writable ray and screen-point arrays (outputs of the two producers). */
typedef struct xk_rays_out {
    double *x, *y, *z, *nx, *ny, *nz, *nl, *es_re, *es_im, *ep_re, *ep_im, *energy;
} xk_rays_out;
typedef struct xk_pixels_out {
    double *x, *y, *z;
} xk_pixels_out;

/* prepare_wave (src/waves/prepare_wave.rs:40-68): the nx*nz screen points,
 * x outer and z inner (index ix*nz + iz), y = center[1], computed on the
 * device with the reference's operation order; `out` holds host arrays of
 * nx*nz doubles. nx*nz == 0 is a no-op. */
int xk_prepare_wave(xk_ctx* ctx, const xk_wave_params* params, xk_pixels_out* out);

/* beam_to_diffraction_rays (src/waves/prepare_wave.rs:78-111): ray i is beam
 * ray good[i] with its surface normal normals[3*good[i] .. +3] and
 * nl = n.(a, b, c); `beam` and `normals` (n_beam rows of 3 doubles) are host
 * arrays, `out` holds host arrays of n_good doubles. A good index >= n_beam
 * returns XK_ERR_INVALID (the reference panics). */
int xk_beam_to_rays(xk_ctx* ctx, const xk_beam* beam, size_t n_beam, const double* normals,
                    const size_t* good, size_t n_good, xk_rays_out* out);

/* The whole chain on the device: uploads the beam's columns, builds the rays
 * of `good` and the screen of `params` in HBM and solves the integral on them
 * (as xk_diffraction_integral, whose result it equals bit for bit). `out`
 * holds host arrays of params->nx * params->nz doubles. */
int xk_diffraction_beam(xk_ctx* ctx, const xk_beam* beam, size_t n_beam, const double* normals,
                        const size_t* good, size_t n_good, const xk_wave_params* params,
                        xk_field* out, int path, xk_stats* stats);

/* ---- 2-D Fresnel propagation ---------------------------------------------
 *
 * waves::fresnel::fresnel_propagate (src/waves/fresnel.rs:53-106): rays at
 * (x_j, z_j) on the source plane with complex amplitude es_j, screen of
 * nx x nz points x_i = x_min + (x_max - x_min) * i / max(nx - 1, 1) (same in
 * z) at distance `dist`, k = energy / CHBAR * 1e7,
 *   U(x, z) = sum_j es_j exp(i k/(2 dist) ((x - x_j)^2 + (z - z_j)^2)),
 * output index iz * nx + ix (z outer, as the reference).
 *
 * Paths:
 *   XK_PATH_F64        the reference's sum in FP64, term for term (parity).
 *   XK_PATH_SEPARABLE  the Fresnel kernel factorises over a regular screen,
 *                      exp(i a r^2) = exp(i a dx^2) exp(i a dz^2), so the
 *                      screen is one complex matrix product over the rays:
 *                      phasors from FP64 phases, split into f16 hi + lo
 *                      parts inside the kernel, multiplied on the tensor
 *                      cores with f32 accumulation (three partial products),
 *                      drained into FP64 every few ray blocks; K-split
 *                      partials added in FP64. */
typedef struct xk_fresnel_screen {
    double x_min, x_max;
    size_t nx;
    double z_min, z_max;
    size_t nz;
} xk_fresnel_screen;

/* Host buffers: rays (n_rays each), amp_re / amp_im (nx * nz each), and
 * optionally x_pixels (nx) and z_pixels (nz), the FresnelResult coordinates
 * (NULL to skip). nx * nz == 0 is a no-op; no rays give zeros. */
int xk_fresnel_propagate(xk_ctx* ctx, const double* ray_x, const double* ray_z,
                         const double* es_re, const double* es_im, size_t n_rays, double energy,
                         double dist, const xk_fresnel_screen* screen, double* amp_re,
                         double* amp_im, double* x_pixels, double* z_pixels, int path,
                         xk_stats* stats);

/* ---- batches of solves ------------------------------------------------------
 *
 * Many independent solves of uneven sizes in one persistent launch. No
 * counterpart in the reference, which solves one problem per call; each
 * solve keeps the semantics of xk_diffraction_integral. */
typedef struct xk_solve {
    xk_rays rays;
    size_t n_rays;
    xk_pixels pixels;
    size_t n_pix;
    xk_field out;
} xk_solve;

enum {
    XK_BATCH_DEVICE = 1,   /* every pointer in the solves is a device pointer */
    XK_BATCH_NO_GRAPH = 2  /* enqueue the launches on each run instead of replaying a graph */
};

typedef struct xk_batch xk_batch;

typedef struct xk_batch_stats {
    double pairs;       /* sum of n_rays * n_pix */
    double plan_ms;     /* host wall time of xk_batch_create (copies + planning) */
    double exec_ms;     /* device time of the run's launches (CUDA events) */
    double wall_ms;     /* host wall time of xk_batch_run incl. output copies */
    int n_solves;
    int routed_f64;     /* solves that ran on XK_PATH_F64 */
    int kernels;        /* kernel launches per run */
    int graph;          /* 1 if the run replayed a CUDA graph */
    long long n_items;  /* FP32-PR work items per run */
} xk_batch_stats;

typedef struct xk_solve_plan {
    int path, routed_reason, n_tiles, n_chunks, groups, sweep;
    double phase_bound_rad;
    int one_polarization;
    int tuned;  /* 1 if the solve uses autotuned settings of its bucket */
} xk_solve_plan;

/* Copies host inputs to the device (unless XK_BATCH_DEVICE), plans every
 * solve in one pass (three host synchronisations for the whole batch) and
 * captures the execution — one persistent launch per kernel variant over all
 * solves' items, then the per-solve reductions — in a CUDA graph. The solves'
 * input and output buffers must stay valid until xk_batch_destroy. */
int xk_batch_create(xk_ctx* ctx, const xk_solve* solves, size_t n, int path, int flags,
                    xk_batch** out);

/* Runs the batch (graph replay) and writes every solve's field to its `out`
 * buffers; blocks until done. Repeated runs recompute the same inputs. */
int xk_batch_run(xk_batch* batch, xk_batch_stats* stats);

/* Plan of solve i (valid after xk_batch_create; chunk counts after a run). */
int xk_batch_solve_plan(const xk_batch* batch, size_t i, xk_solve_plan* out);

void xk_batch_destroy(xk_batch* batch);

/* ---- serving: continuous batching --------------------------------------------
 *
 * No counterpart in the reference (one blocking call per solve). A server
 * accepts solves from any thread; a worker admits them while the admitted
 * set fits an HBM budget, plans them, and runs them in epochs: each epoch is
 * one persistent launch over work items of every admitted request (a fair
 * share each), so a request that arrives while others run joins the next
 * epoch. A request's result does not depend on what else is in flight. */
typedef struct xk_server xk_server;

typedef struct xk_server_opts {
    double hbm_budget_bytes;          /* admission budget; 0 = 120e9 */
    double epoch_pairs;               /* ray x screen pairs per epoch; 0 = 3e10 */
    int max_active;                   /* admitted requests at once; 0 = 64 */
    double item_pairs;                /* target pairs per work item; 0 = 1e6 */
    int inject_alloc_failure_every;   /* testing: fail every k-th request allocation; 0 = off */
    int reserve_sms;                  /* SMs epochs leave free for planning kernels; 0 = 8 */
    int policy;                       /* how an epoch's pair budget is shared among running
                                         requests: XK_SERVE_SHORTEST_AGED (0, default) fills it in
                                         order of remaining pairs / (1 + waited / aging_ms), so
                                         small requests finish in few epochs and the wait of
                                         large ones stays bounded; XK_SERVE_EQUAL_SHARE (1) gives
                                         every running request the same share */
    double aging_ms;                  /* aging constant of XK_SERVE_SHORTEST_AGED; 0 = 1000 */
} xk_server_opts;

#define XK_SERVE_SHORTEST_AGED 0
#define XK_SERVE_EQUAL_SHARE 1

typedef struct xk_request {
    xk_rays rays;       /* host pointers; ignored when rayset != 0 */
    size_t n_rays;
    uint64_t rayset;    /* handle from xk_server_upload_rays, 0 = use `rays` */
    xk_pixels pixels;   /* host pointers */
    size_t n_pix;       /* > 0 */
    xk_field out;       /* host pointers, written before the request completes */
    int path;           /* XK_PATH_F32PR or XK_PATH_F64 */
} xk_request;

typedef struct xk_request_stats {
    double pairs;
    double queue_ms;    /* submit -> admitted */
    double plan_ms;     /* admitted -> planned (copies + planning) */
    double run_ms;      /* planned -> result on the host */
    double total_ms;    /* submit -> result on the host */
    int path;           /* path actually used */
    int epochs;         /* epochs that ran this request's items */
    int status;
} xk_request_stats;

typedef struct xk_server_stats {
    long long submitted, completed, failed, epochs, kernels, pending, active;
    double pairs_done, used_bytes, peak_bytes, resident_ray_bytes;
    double pairs_launched;  /* ray x screen pairs of all work items launched so far */
} xk_server_stats;

int xk_server_create(xk_ctx* ctx, const xk_server_opts* opts, xk_server** out);

/* Copies a ray set to the device and keeps it there for any number of
 * requests (screens) until released; it counts against the budget. */
int xk_server_upload_rays(xk_server* server, const xk_rays* rays, size_t n, uint64_t* handle);
int xk_server_release_rays(xk_server* server, uint64_t handle);

/* A resident ray set built on the device straight from a beam: the columns of
 * `beam`, its normals and `good` (host arrays, as xk_beam_to_rays) go to the
 * GPU once and beam_to_diffraction_rays (src/waves/prepare_wave.rs:78-111)
 * runs there, so the n_good ray records never exist on the host. Released
 * with xk_server_release_rays. A good index >= n_beam returns XK_ERR_INVALID. */
int xk_server_upload_beam(xk_server* server, const xk_beam* beam, size_t n_beam,
                          const double* normals, const size_t* good, size_t n_good,
                          uint64_t* handle);

/* Queues a request; its host buffers must stay valid until xk_server_wait
 * returns for the ticket. Returns at once. */
int xk_server_submit(xk_server* server, const xk_request* req, uint64_t* ticket);

/* Blocks until the request completes (timeout_ms < 0: no limit; on time-out
 * returns XK_ERR_TIMEOUT and the ticket stays valid). Returns the request's
 * own status (XK_ERR_BUDGET if it alone exceeds the budget, XK_ERR_SHUTDOWN if
 * the server stopped before admitting it) and releases the ticket. */
int xk_server_wait(xk_server* server, uint64_t ticket, double timeout_ms,
                   xk_request_stats* stats);

int xk_server_get_stats(xk_server* server, xk_server_stats* out);

/* Stops: waits for the epochs already launched, then cancels every request
 * not yet completed (their waits return XK_ERR_SHUTDOWN) and frees the server.
 * Tickets are invalid afterwards. */
void xk_server_destroy(xk_server* server);

/* ---- allocation-free FP64 solve ---------------------------------------------
 *
 * No counterpart in the reference. For callers that cannot let a library
 * allocate device memory: programs whose device memory is all owned by their
 * own pool allocator, and loops that cannot pay for cudaMalloc's implicit
 * synchronisation on every call. It runs the kernels of XK_PATH_F64 with
 * its scratch in a fixed array inside the library instead of context buffers,
 * and it calls no cudaMalloc, cudaFree or other allocating routine. Its
 * split-ray partial sums must fit that array, so on solves of more than
 * about 2^24 ray x screen pairs it may cut the ray list into fewer ranges
 * than XK_PATH_F64 does (one range above 524288 screen points); the Kahan
 * sums then run
 * in another order, and results agree with XK_PATH_F64 to <= 1e-10 relative
 * L2 rather than bit for bit.
 *
 * - rays, pixels and out hold DEVICE pointers on the current device; the
 *   work is enqueued on `stream` (cudaStream_t, NULL = default stream) and
 *   the results are ready once that stream is synchronised.
 * - n_rays may not exceed XK_NOALLOC_MAX_RAYS: larger requests return
 *   XK_ERR_BUDGET and launch nothing. n_pix is not limited.
 * - The fixed scratch is XK_NOALLOC_SCRATCH_BYTES (32 MiB) of device memory,
 *   held by every GPU on which the library's FP64 code is loaded until exit.
 * - The first call on a device looks up the scratch's device address with
 *   that device current, and so does the first call after the device's
 *   context was replaced (cudaDeviceReset); make those calls before any
 *   stream capture.
 * - All calls share the one scratch array and it keeps the last call's
 *   contents (every byte a call reads is written earlier in the same call, so
 *   nothing needs clearing). Calls that overlap on the GPU — from several
 *   host threads, or on several streams without ordering between them — race
 *   on the scratch and corrupt each other's results: serialise them. */
#define XK_NOALLOC_MAX_RAYS 131072
#define XK_NOALLOC_SCRATCH_BYTES (32u << 20)
int xk_diffraction_f64_noalloc(const xk_rays* rays, size_t n_rays, const xk_pixels* pixels,
                               size_t n_pix, xk_field* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* XK_H */
