// C-ABI entry points of the xk library (declared in include/xk.h).
//
// The context mirrors gpu::context::GpuContext (src/gpu/context.rs): one per
// device, a process-wide shared instance, the device name. Calls that take
// host buffers stage them through device buffers the context keeps and
// grows, so repeated calls of the same size allocate nothing.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "xk_ctx.cuh"

namespace {

const char* kVersion = "xk 0.1.0 (sm_100a)";

int fail(xk_ctx* ctx, const xk::Status& st) {
    if (ctx) ctx->last_error = st.msg;
    return st.code;
}

int fail(xk_ctx* ctx, int code, const char* msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

xk::Status create_ctx(int device, xk_ctx** out) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();  // clear the sticky "no device" state
        return xk::Status::Err(XK_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count)
        return xk::Status::Err(XK_ERR_INVALID, "device index out of range");
    XK_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    XK_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    xk_ctx* ctx = new xk_ctx();
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    ctx->name = prop.name;
    ctx->pr_opts.tune = &ctx->tune;
    cudaError_t e1 = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    cudaError_t e2 = cudaEventCreate(&ctx->ev0);
    cudaError_t e3 = cudaEventCreate(&ctx->ev1);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
        delete ctx;
        return xk::Status::Err(XK_ERR_CUDA, "stream/event creation failed");
    }
    *out = ctx;
    return xk::Status::Ok();
}

void destroy_ctx(xk_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->f64ws.rays.release();
    ctx->f64ws.partials.release();
    ctx->prws.release();
    ctx->in_rays.release();
    ctx->in_pix.release();
    ctx->out_field.release();
    ctx->in_beam.release();
    ctx->fresnel.coords.release();
    ctx->fresnel.partial.release();
    ctx->fresnel.ctrl.release();
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

bool rays_ok(const xk_rays* r) {
    return r && r->x && r->y && r->z && r->nx && r->ny && r->nz && r->nl && r->es_re &&
           r->es_im && r->ep_re && r->ep_im && r->energy;
}
bool pix_ok(const xk_pixels* p) { return p && p->x && p->y && p->z; }
bool field_ok(const xk_field* f) { return f && f->es_re && f->es_im && f->ep_re && f->ep_im; }

xk::RaysDev to_dev(const xk_rays* r) {
    return xk::RaysDev{r->x, r->y, r->z, r->nx, r->ny, r->nz, r->nl,
                       r->es_re, r->es_im, r->ep_re, r->ep_im, r->energy};
}

// Runs one solve on device data; records events around the compute and
// returns after the stream is synchronised.
xk::Status run_solve(xk_ctx* ctx, const xk::RaysDev& rays, size_t n_rays, const xk::PixDev& pix,
                     size_t n_pix, const xk::FieldDev& out, int path, cudaStream_t stream,
                     xk_stats* stats, int* used_path) {
    xk::NvtxRange nvtx_range("xk solve");
    xk::LaunchReport rep;
    XK_CUDA_TRY(cudaEventRecord(ctx->ev0, stream));
    int used = path;
    if (path == XK_PATH_F32PR) {
        std::vector<xk::PrPlan> plans;
        xk::PrSolveIn in{rays, n_rays, pix, n_pix, out};
        int nk = 0;
        XK_TRY(xk::pr_plan(&in, 1, ctx->prws, stream, ctx->num_sms, ctx->pr_opts, plans, &nk));
        rep.kernels += nk;
        xk::PrPlan& P = plans[0];
        xk::PrExecReport er;
        if (P.routed) {
            used = XK_PATH_F64;
            XK_TRY(xk::f64_enqueue(rays, n_rays, pix, n_pix, out, ctx->f64ws, stream, ctx->num_sms,
                                   &rep));
        } else {
            XK_TRY(xk::pr_execute_enqueue(plans, ctx->prws, stream, ctx->num_sms, true, &er));
            rep.kernels += er.kernels;
        }
        XK_CUDA_TRY(cudaEventRecord(ctx->ev1, stream));
        XK_CUDA_TRY(cudaStreamSynchronize(stream));
        if (!P.routed) XK_TRY(xk::pr_execute_finish(plans, ctx->prws, &er));
        ctx->last_energy_ev = P.energy_ev;
        ctx->last_dist_mm = P.dist_mm;
        if (stats) {
            stats->tuned = P.tuned ? 1 : 0;
            stats->folded = !P.routed && P.fold ? 1 : 0;
            stats->n_tiles = P.n_tiles;
            stats->n_chunks = P.n_chunks;
            stats->n_items = (long long)P.n_tiles * P.groups;
            stats->phase_bound_rad = P.phase_bound;
            stats->groups = P.groups;
            stats->routed_reason = P.routed ? P.route_reason : 0;
            stats->main_kernel_ms = er.main_kernel_ms;
            stats->sweep = P.routed ? -1 : (P.fast ? (P.lin ? 2 : 1) : 0);
            stats->one_polarization = !P.routed && P.one_pol;
        }
    } else {
        XK_TRY(xk::f64_enqueue(rays, n_rays, pix, n_pix, out, ctx->f64ws, stream, ctx->num_sms,
                               &rep));
        XK_CUDA_TRY(cudaEventRecord(ctx->ev1, stream));
        XK_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    if (stats) stats->kernels += rep.kernels;
    *used_path = used;
    return xk::Status::Ok();
}

xk::Status finish_stats(xk_ctx* ctx, xk_stats* stats, int used_path, size_t n_rays,
                        size_t n_pix) {
    if (!stats) return xk::Status::Ok();
    float ms = 0.f;
    XK_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    stats->gpu_ms = ms;
    stats->path = used_path;
    stats->pairs = (double)n_rays * (double)n_pix;
    return xk::Status::Ok();
}

xk::Status solve_host(xk_ctx* ctx, const xk_rays* rays, size_t n_rays, const xk_pixels* pixels,
                      size_t n_pix, xk_field* out, int path, xk_stats* stats) {
    cudaStream_t s = ctx->stream;
    const size_t nb = n_rays * sizeof(double), mb = n_pix * sizeof(double);
    XK_TRY(ctx->in_rays.ensure(12 * nb > 0 ? 12 * nb : 8));
    XK_TRY(ctx->in_pix.ensure(3 * mb));
    XK_TRY(ctx->out_field.ensure(4 * mb));
    double* dr = ctx->in_rays.as<double>();
    const double* hsrc[12] = {rays->x, rays->y, rays->z, rays->nx, rays->ny, rays->nz,
                              rays->nl, rays->es_re, rays->es_im, rays->ep_re, rays->ep_im,
                              rays->energy};
    for (int i = 0; i < 12 && n_rays; ++i)
        XK_CUDA_TRY(cudaMemcpyAsync(dr + i * n_rays, hsrc[i], nb, cudaMemcpyHostToDevice, s));
    double* dp = ctx->in_pix.as<double>();
    XK_CUDA_TRY(cudaMemcpyAsync(dp, pixels->x, mb, cudaMemcpyHostToDevice, s));
    XK_CUDA_TRY(cudaMemcpyAsync(dp + n_pix, pixels->y, mb, cudaMemcpyHostToDevice, s));
    XK_CUDA_TRY(cudaMemcpyAsync(dp + 2 * n_pix, pixels->z, mb, cudaMemcpyHostToDevice, s));
    xk::RaysDev rd;
    const double** f = reinterpret_cast<const double**>(&rd);
    for (int i = 0; i < 12; ++i) f[i] = dr + i * n_rays;
    xk::PixDev pd{dp, dp + n_pix, dp + 2 * n_pix};
    double* dout = ctx->out_field.as<double>();
    xk::FieldDev fd{dout, dout + n_pix, dout + 2 * n_pix, dout + 3 * n_pix};
    int used = path;
    XK_TRY(run_solve(ctx, rd, n_rays, pd, n_pix, fd, path, s, stats, &used));
    double* hdst[4] = {out->es_re, out->es_im, out->ep_re, out->ep_im};
    for (int i = 0; i < 4; ++i)
        XK_CUDA_TRY(cudaMemcpyAsync(hdst[i], dout + i * n_pix, mb, cudaMemcpyDeviceToHost, s));
    XK_CUDA_TRY(cudaStreamSynchronize(s));
    if (stats) {
        stats->h2d_bytes = 12.0 * nb + 3.0 * mb;
        stats->d2h_bytes = 4.0 * mb;
    }
    return finish_stats(ctx, stats, used, n_rays, n_pix);
}


// ---- screen grid and beam producers ---------------------------------------

static_assert(sizeof(size_t) == sizeof(uint64_t), "good indices are copied as 64-bit words");

bool beam_ok(const xk_beam* b) {
    if (!b || !b->x || !b->y || !b->z || !b->a || !b->b || !b->c || !b->e) return false;
    const int amps = !!b->es_re + !!b->es_im + !!b->ep_re + !!b->ep_im;
    return amps == 0 || amps == 4;
}

xk::Status wave_size(const xk_wave_params* p, size_t* m) {
    if (p->nx && p->nz > SIZE_MAX / p->nx)
        return xk::Status::Err(XK_ERR_INVALID, "nx * nz overflows");
    *m = p->nx * p->nz;
    return xk::Status::Ok();
}

xk::WaveGrid to_grid(const xk_wave_params* p) {
    return xk::WaveGrid{p->center[0], p->center[1], p->center[2], p->dx, p->dz, p->nx, p->nz};
}

// Uploads the beam columns, normals and good indices into ctx->in_beam.
xk::Status upload_beam(xk_ctx* ctx, const xk_beam* beam, size_t n_beam, const double* normals,
                       const size_t* good, size_t n_good, cudaStream_t s, xk::BeamDev* bd,
                       const uint64_t** d_good, double* h2d) {
    for (size_t i = 0; i < n_good; ++i)
        if (good[i] >= n_beam) return xk::Status::Err(XK_ERR_INVALID, "good index out of range");
    const bool amps = beam->es_re != nullptr;
    const int cols = amps ? 11 : 7;
    const size_t nb = n_beam * sizeof(double);
    const size_t bytes = (size_t)cols * nb + 3 * nb + n_good * sizeof(uint64_t);
    XK_TRY(ctx->in_beam.ensure(std::max<size_t>(bytes, 8)));
    double* d = ctx->in_beam.as<double>();
    const double* src[11] = {beam->x, beam->y, beam->z, beam->a, beam->b, beam->c, beam->e,
                             beam->es_re, beam->es_im, beam->ep_re, beam->ep_im};
    const double** dst = reinterpret_cast<const double**>(bd);
    *bd = xk::BeamDev{};
    for (int f = 0; f < cols; ++f) {
        dst[f] = d;
        if (n_beam) XK_CUDA_TRY(cudaMemcpyAsync(d, src[f], nb, cudaMemcpyHostToDevice, s));
        d += n_beam;
    }
    bd->normals = d;
    if (n_beam) XK_CUDA_TRY(cudaMemcpyAsync(d, normals, 3 * nb, cudaMemcpyHostToDevice, s));
    d += 3 * n_beam;
    *d_good = reinterpret_cast<const uint64_t*>(d);
    if (n_good)
        XK_CUDA_TRY(cudaMemcpyAsync(d, good, n_good * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    *h2d = (double)bytes;
    return xk::Status::Ok();
}

// Device columns of the ray staging buffer (12 x n).
void ray_columns(xk_ctx* ctx, size_t n, double* cols[12], xk::RaysDev* rd) {
    double* d = ctx->in_rays.as<double>();
    const double** f = reinterpret_cast<const double**>(rd);
    for (int i = 0; i < 12; ++i) {
        cols[i] = d + i * n;
        f[i] = cols[i];
    }
}

}  // namespace

extern "C" {

const char* xk_version(void) { return kVersion; }

const char* xk_route_reason(int reason) {
    if (reason < 0 || reason >= xk::kRouteReasonCount) return "unknown";
    return xk::kRouteReasons[reason];
}

const char* xk_status_string(int status) {
    switch (status) {
        case XK_OK: return "ok";
        case XK_ERR_NO_DEVICE: return "no CUDA device";
        case XK_ERR_INVALID: return "invalid argument";
        case XK_ERR_OOM: return "out of memory";
        case XK_ERR_BUDGET: return "request exceeds the HBM budget";
        case XK_ERR_CUDA: return "CUDA error";
        case XK_ERR_TIMEOUT: return "timed out";
        case XK_ERR_NOT_FOUND: return "unknown handle or ticket";
        case XK_ERR_CANCELLED: return "cancelled";
        case XK_ERR_SHUTDOWN: return "server shutting down";
        default: return "unknown status";
    }
}

int xk_init(int device, xk_ctx** out) {
    if (!out) return XK_ERR_INVALID;
    *out = nullptr;
    xk::Status st = create_ctx(device, out);
    return st.code;
}

int xk_shared(xk_ctx** out) {
    static std::once_flag once;
    static xk_ctx* shared = nullptr;
    static int shared_status = XK_OK;
    if (!out) return XK_ERR_INVALID;
    std::call_once(once, [] {
        xk_ctx* c = nullptr;
        xk::Status st = create_ctx(0, &c);
        shared_status = st.code;
        if (st.ok()) {
            c->is_shared = true;
            shared = c;
        }
    });
    *out = shared;
    return shared ? XK_OK : shared_status;
}

void xk_destroy(xk_ctx* ctx) {
    if (!ctx || ctx->is_shared) return;
    destroy_ctx(ctx);
}

const char* xk_device_name(const xk_ctx* ctx) { return ctx ? ctx->name.c_str() : ""; }

const char* xk_last_error(const xk_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int xk_set_option(xk_ctx* ctx, const char* name, double value) {
    if (!ctx || !name) return XK_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string n(name);
    if (n == "phase_budget") {
        if (!(value > 0.0) || value > 1e5) return fail(ctx, XK_ERR_INVALID, "phase_budget out of range");
        ctx->pr_opts.phase_budget = value;
    } else if (n == "tolerance") {
        if (!(value >= 1e-7) || value > 1e-2)
            return fail(ctx, XK_ERR_INVALID, "tolerance must be in [1e-7, 1e-2]");
        ctx->pr_opts.tolerance = value;
    } else if (n == "sweep") {
        if (value != -1.0 && value != 0.0 && value != 1.0 && value != 2.0)
            return fail(ctx, XK_ERR_INVALID, "sweep must be -1, 0, 1 or 2");
        ctx->pr_opts.sweep = (int)value;
    } else if (n == "groups") {
        if (value < 0.0 || value > 65536.0) return fail(ctx, XK_ERR_INVALID, "groups out of range");
        ctx->pr_opts.groups = (int)value;
    } else if (n == "f64_reduction") {
        if (value != 0.0 && value != 1.0) return fail(ctx, XK_ERR_INVALID, "f64_reduction is 0 or 1");
        ctx->f64ws.fast_reduction = value != 0.0;
    } else if (n == "polarization") {
        if (value != -1.0 && value != 0.0)
            return fail(ctx, XK_ERR_INVALID, "polarization must be -1 or 0");
        ctx->pr_opts.polarization = (int)value;
    } else if (n == "items_per_warp") {
        if (value < 1.0 || value > 4096.0) return fail(ctx, XK_ERR_INVALID, "items_per_warp out of range");
        ctx->pr_opts.items_per_warp = (long long)value;
    } else if (n == "use_tuned") {
        if (value != 0.0 && value != 1.0) return fail(ctx, XK_ERR_INVALID, "use_tuned is 0 or 1");
        ctx->tune.use = value != 0.0;
    } else if (n == "clear_tuned") {
        ctx->tune.clear();
    } else if (n == "wait_limit") {
        if (!(value >= 1.0) || value > 2147483648.0 || value != std::floor(value))
            return fail(ctx, XK_ERR_INVALID, "wait_limit must be an integer in 1..2^31");
        ctx->prws.ctl.wait_limit = (uint32_t)value;
        ctx->fresnel.wait_limit = (uint32_t)value;
    } else if (n == "fresnel_pair") {
        if (value != 0.0 && value != 1.0) return fail(ctx, XK_ERR_INVALID, "fresnel_pair is 0 or 1");
        ctx->fresnel.allow_pair = value != 0.0;
    } else if (n == "fresnel_stall") {
        if (value != 0.0 && value != 1.0) return fail(ctx, XK_ERR_INVALID, "fresnel_stall is 0 or 1");
        ctx->fresnel.stall_once = (uint32_t)value;
    } else if (n == "inject_stall") {
        if (!(value >= 0.0) || value > 1024.0 || std::fmod(value, 16.0) != 0.0)
            return fail(ctx, XK_ERR_INVALID, "inject_stall must be a multiple of 16 in 0..1024");
        ctx->prws.ctl.stall_bytes = (uint32_t)value;
    } else {
        return fail(ctx, XK_ERR_INVALID, "unknown option");
    }
    return XK_OK;
}

int xk_autotune(xk_ctx* ctx, const xk_rays* rays, size_t n_rays, const xk_pixels* pixels,
                size_t n_pix, xk_field* out, double budget_ms, int apply,
                xk_tune_result* result) {
    if (!ctx || !result) return XK_ERR_INVALID;
    if (!rays_ok(rays) || !pix_ok(pixels) || !field_ok(out) || n_rays == 0 || n_pix == 0)
        return fail(ctx, XK_ERR_INVALID, "autotune needs a non-empty device-resident problem");
    std::memset(result, 0, sizeof(*result));
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    const xk::RaysDev rd = to_dev(rays);
    const xk::PixDev pd{pixels->x, pixels->y, pixels->z};
    const xk::FieldDev fd{out->es_re, out->es_im, out->ep_re, out->ep_im};
    const xk::PrOptions base = ctx->pr_opts;
    // Candidates: the defaults first, then larger and smaller residual-phase
    // budgets (ray chunks grow with the budget; the tolerance caps it, so no
    // candidate loosens the error bound), more or fewer items per warp, and
    // the sweeps. Trials ignore the tuning cache.
    struct Cand {
        double budget;
        long long ipw;
        int sweep;
    };
    const Cand cands[] = {{base.phase_budget, base.items_per_warp, base.sweep},
                          {512.0, 32, -1}, {512.0, 8, -1}, {192.0, 16, -1}, {384.0, 16, -1},
                          {512.0, 16, 1},  {512.0, 16, 0}, {192.0, 32, -1}, {192.0, 8, -1},
                          {128.0, 16, -1}, {512.0, 4, -1}, {96.0, 16, -1}};
    double spent = 0.0, best = 1e300;
    xk::PrOptions best_opt = base;
    int trials = 0;
    for (const Cand& c : cands) {
        if (trials > 0 && spent >= budget_ms) break;
        ctx->pr_opts = base;
        ctx->pr_opts.tune = nullptr;
        ctx->pr_opts.phase_budget = std::min(c.budget, base.phase_budget);
        ctx->pr_opts.items_per_warp = c.ipw;
        ctx->pr_opts.sweep = c.sweep;
        xk_stats st;
        std::memset(&st, 0, sizeof(st));
        int used = XK_PATH_F32PR;
        xk::Status s = run_solve(ctx, rd, n_rays, pd, n_pix, fd, XK_PATH_F32PR, ctx->stream, &st, &used);
        if (s.ok()) s = finish_stats(ctx, &st, used, n_rays, n_pix);
        if (!s.ok()) {
            ctx->pr_opts = base;
            return fail(ctx, s);
        }
        ++trials;
        spent += st.gpu_ms;
        if (trials == 1) result->default_ms = st.gpu_ms;
        if (used != XK_PATH_F32PR) break;  // routed to FP64: nothing to tune
        if (st.gpu_ms < best) {
            best = st.gpu_ms;
            best_opt = ctx->pr_opts;
        }
    }
    ctx->pr_opts = base;
    if (apply && trials > 0 && best < 1e299) {
        // Kept for this problem's bucket; the context's own defaults stay.
        xk::PrTuned t;
        t.phase_budget = best_opt.phase_budget;
        t.items_per_warp = best_opt.items_per_warp;
        t.sweep = best_opt.sweep;
        ctx->tune.store(ctx->last_energy_ev, ctx->last_dist_mm, n_rays, n_pix, t);
    }
    result->best_ms = best < 1e299 ? best : result->default_ms;
    result->phase_budget = best_opt.phase_budget;
    result->items_per_warp = best_opt.items_per_warp;
    result->sweep = best_opt.sweep;
    result->trials = trials;
    return XK_OK;
}

int xk_diffraction_integral(xk_ctx* ctx, const xk_rays* rays, size_t n_rays,
                            const xk_pixels* pixels, size_t n_pix, xk_field* out, int path,
                            xk_stats* stats) {
    if (!ctx) return XK_ERR_INVALID;
    if ((n_rays && !rays_ok(rays)) || (n_pix && (!pix_ok(pixels) || !field_ok(out))))
        return fail(ctx, XK_ERR_INVALID, "null array pointer");
    if (path != XK_PATH_F64 && path != XK_PATH_F32PR)
        return fail(ctx, XK_ERR_INVALID, "unknown path");
    auto t0 = std::chrono::steady_clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (n_pix == 0) return XK_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    xk::Status st = solve_host(ctx, rays, n_rays, pixels, n_pix, out, path, stats);
    if (!st.ok()) return fail(ctx, st);
    if (stats)
        stats->wall_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                .count();
    return XK_OK;
}

int xk_diffraction_integral_device(xk_ctx* ctx, const xk_rays* rays, size_t n_rays,
                                   const xk_pixels* pixels, size_t n_pix, xk_field* out,
                                   int path, void* stream, xk_stats* stats) {
    if (!ctx) return XK_ERR_INVALID;
    if ((n_rays && !rays_ok(rays)) || (n_pix && (!pix_ok(pixels) || !field_ok(out))))
        return fail(ctx, XK_ERR_INVALID, "null array pointer");
    if (path != XK_PATH_F64 && path != XK_PATH_F32PR)
        return fail(ctx, XK_ERR_INVALID, "unknown path");
    auto t0 = std::chrono::steady_clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (n_pix == 0) return XK_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    xk::RaysDev rd{};
    if (n_rays) rd = to_dev(rays);
    xk::PixDev pd{pixels->x, pixels->y, pixels->z};
    xk::FieldDev fd{out->es_re, out->es_im, out->ep_re, out->ep_im};
    int used = path;
    xk::Status st = run_solve(ctx, rd, n_rays, pd, n_pix, fd, path, s, stats, &used);
    if (st.ok()) st = finish_stats(ctx, stats, used, n_rays, n_pix);
    if (!st.ok()) return fail(ctx, st);
    if (stats)
        stats->wall_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                .count();
    return XK_OK;
}

int xk_kirchhoff_gpu(xk_ctx* ctx, const xk_gpu_ray* rays, size_t n_rays,
                     const xk_gpu_pixel* pixels, size_t n_pix, double* out) {
    if (!ctx) return XK_ERR_INVALID;
    if ((n_rays && !rays) || (n_pix && (!pixels || !out)))
        return fail(ctx, XK_ERR_INVALID, "null pointer");
    if (n_pix == 0) return XK_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    // The f32 records go to the device as they are (48 + 16 bytes each) and
    // are widened to f64 SoA there (exact, as the reference's host side
    // promotes them for the base-phase restore, kirchhoff.rs:96-104); the
    // field comes back as 4 doubles per pixel.
    const size_t rec_bytes = n_rays * sizeof(xk_gpu_ray), pix_bytes = n_pix * sizeof(xk_gpu_pixel);
    const size_t rec_off = 0, pix_off = (rec_bytes + 255) / 256 * 256;
    const size_t out_off = pix_off + (pix_bytes + 255) / 256 * 256;
    xk::Status st = ctx->in_beam.ensure(out_off + 4 * n_pix * sizeof(double));
    if (st.ok()) st = ctx->in_rays.ensure(std::max<size_t>(12 * n_rays * sizeof(double), 8));
    if (st.ok()) st = ctx->in_pix.ensure(3 * n_pix * sizeof(double));
    if (st.ok()) st = ctx->out_field.ensure(4 * n_pix * sizeof(double));
    if (!st.ok()) return fail(ctx, st);
    char* staging = ctx->in_beam.as<char>();
    auto* d_rec = reinterpret_cast<xk_gpu_ray*>(staging + rec_off);
    auto* d_pxr = reinterpret_cast<xk_gpu_pixel*>(staging + pix_off);
    double* d_out = reinterpret_cast<double*>(staging + out_off);
    if (n_rays)
        st = xk::Status::FromCuda(
            cudaMemcpyAsync(d_rec, rays, rec_bytes, cudaMemcpyHostToDevice, s));
    if (st.ok())
        st = xk::Status::FromCuda(
            cudaMemcpyAsync(d_pxr, pixels, pix_bytes, cudaMemcpyHostToDevice, s));
    double* cols[12];
    xk::RaysDev rd;
    ray_columns(ctx, n_rays, cols, &rd);
    double* dp = ctx->in_pix.as<double>();
    if (st.ok()) st = xk::gpu_records_enqueue(d_rec, n_rays, d_pxr, n_pix, cols, dp, dp + n_pix,
                                              dp + 2 * n_pix, s);
    xk::PixDev pd{dp, dp + n_pix, dp + 2 * n_pix};
    double* dout = ctx->out_field.as<double>();
    xk::FieldDev fd{dout, dout + n_pix, dout + 2 * n_pix, dout + 3 * n_pix};
    int used = XK_PATH_F32PR;
    if (st.ok()) st = run_solve(ctx, rd, n_rays, pd, n_pix, fd, XK_PATH_F32PR, s, nullptr, &used);
    if (st.ok()) st = xk::interleave_field_enqueue(fd, n_pix, d_out, s);
    if (st.ok()) st = xk::Status::FromCuda(cudaMemcpyAsync(out, d_out, 4 * n_pix * sizeof(double),
                                                           cudaMemcpyDeviceToHost, s));
    if (st.ok()) st = xk::Status::FromCuda(cudaStreamSynchronize(s));
    return st.ok() ? XK_OK : fail(ctx, st);
}

int xk_kirchhoff_auto(const xk_gpu_ray* rays, size_t n_rays, const xk_gpu_pixel* pixels,
                      size_t n_pix, double* out) {
    xk_ctx* ctx = nullptr;
    int rc = xk_shared(&ctx);
    if (rc != XK_OK || !ctx) return rc == XK_OK ? XK_ERR_NO_DEVICE : rc;
    return xk_kirchhoff_gpu(ctx, rays, n_rays, pixels, n_pix, out);
}

int xk_prepare_wave(xk_ctx* ctx, const xk_wave_params* params, xk_pixels_out* out) {
    if (!ctx) return XK_ERR_INVALID;
    if (!params) return fail(ctx, XK_ERR_INVALID, "null wave parameters");
    size_t m = 0;
    xk::Status st = wave_size(params, &m);
    if (!st.ok()) return fail(ctx, st);
    if (m == 0) return XK_OK;
    if (!out || !out->x || !out->y || !out->z)
        return fail(ctx, XK_ERR_INVALID, "null array pointer");
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t mb = m * sizeof(double);
    st = ctx->in_pix.ensure(3 * mb);
    if (st.ok()) {
        double* d = ctx->in_pix.as<double>();
        st = xk::wave_enqueue(to_grid(params), d, d + m, d + 2 * m, s);
        double* dst[3] = {out->x, out->y, out->z};
        for (int f = 0; f < 3 && st.ok(); ++f)
            if (cudaMemcpyAsync(dst[f], d + f * m, mb, cudaMemcpyDeviceToHost, s) != cudaSuccess)
                st = xk::Status::Err(XK_ERR_CUDA, "device-to-host copy failed");
        if (st.ok() && cudaStreamSynchronize(s) != cudaSuccess)
            st = xk::Status::Err(XK_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    }
    return st.ok() ? XK_OK : fail(ctx, st);
}

int xk_beam_to_rays(xk_ctx* ctx, const xk_beam* beam, size_t n_beam, const double* normals,
                    const size_t* good, size_t n_good, xk_rays_out* out) {
    if (!ctx) return XK_ERR_INVALID;
    if (n_good == 0) return XK_OK;
    bool out_ok = out != nullptr;
    if (out_ok) {
        double* h[12] = {out->x, out->y, out->z, out->nx, out->ny, out->nz, out->nl,
                         out->es_re, out->es_im, out->ep_re, out->ep_im, out->energy};
        for (double* p : h) out_ok = out_ok && p;
    }
    if (!beam_ok(beam) || !normals || !good || !out_ok)
        return fail(ctx, XK_ERR_INVALID, "null array pointer (or amplitudes only partly set)");
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    xk::BeamDev bd;
    const uint64_t* d_good = nullptr;
    double h2d = 0.0;
    xk::Status st = upload_beam(ctx, beam, n_beam, normals, good, n_good, s, &bd, &d_good, &h2d);
    if (st.ok()) st = ctx->in_rays.ensure(12 * n_good * sizeof(double));
    if (st.ok()) {
        double* cols[12];
        xk::RaysDev rd;
        ray_columns(ctx, n_good, cols, &rd);
        st = xk::beam_rays_enqueue(bd, d_good, n_good, cols, s);
        double* h[12] = {out->x, out->y, out->z, out->nx, out->ny, out->nz, out->nl,
                         out->es_re, out->es_im, out->ep_re, out->ep_im, out->energy};
        for (int f = 0; f < 12 && st.ok(); ++f)
            if (cudaMemcpyAsync(h[f], cols[f], n_good * sizeof(double),
                                cudaMemcpyDeviceToHost, s) != cudaSuccess)
                st = xk::Status::Err(XK_ERR_CUDA, "device-to-host copy failed");
        if (st.ok() && cudaStreamSynchronize(s) != cudaSuccess)
            st = xk::Status::Err(XK_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    }
    return st.ok() ? XK_OK : fail(ctx, st);
}

int xk_diffraction_beam(xk_ctx* ctx, const xk_beam* beam, size_t n_beam, const double* normals,
                        const size_t* good, size_t n_good, const xk_wave_params* params,
                        xk_field* out, int path, xk_stats* stats) {
    if (!ctx) return XK_ERR_INVALID;
    if (!params) return fail(ctx, XK_ERR_INVALID, "null wave parameters");
    if (path != XK_PATH_F64 && path != XK_PATH_F32PR)
        return fail(ctx, XK_ERR_INVALID, "unknown path");
    size_t m = 0;
    xk::Status st = wave_size(params, &m);
    if (!st.ok()) return fail(ctx, st);
    auto t0 = std::chrono::steady_clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (m == 0) return XK_OK;
    if (!field_ok(out) || (n_good && (!beam_ok(beam) || !normals || !good)))
        return fail(ctx, XK_ERR_INVALID, "null array pointer (or amplitudes only partly set)");
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    xk::BeamDev bd;
    const uint64_t* d_good = nullptr;
    double h2d = 0.0;
    if (n_good) st = upload_beam(ctx, beam, n_beam, normals, good, n_good, s, &bd, &d_good, &h2d);
    if (st.ok()) st = ctx->in_rays.ensure(std::max<size_t>(12 * n_good * sizeof(double), 8));
    if (st.ok()) st = ctx->in_pix.ensure(3 * m * sizeof(double));
    if (st.ok()) st = ctx->out_field.ensure(4 * m * sizeof(double));
    if (!st.ok()) return fail(ctx, st);
    double* cols[12];
    xk::RaysDev rd;
    ray_columns(ctx, n_good, cols, &rd);
    st = xk::beam_rays_enqueue(bd, d_good, n_good, cols, s);
    double* dp = ctx->in_pix.as<double>();
    if (st.ok()) st = xk::wave_enqueue(to_grid(params), dp, dp + m, dp + 2 * m, s);
    xk::PixDev pd{dp, dp + m, dp + 2 * m};
    double* dout = ctx->out_field.as<double>();
    xk::FieldDev fd{dout, dout + m, dout + 2 * m, dout + 3 * m};
    int used = path;
    if (st.ok()) st = run_solve(ctx, rd, n_good, pd, m, fd, path, s, stats, &used);
    double* hdst[4] = {out->es_re, out->es_im, out->ep_re, out->ep_im};
    for (int i = 0; i < 4 && st.ok(); ++i)
        if (cudaMemcpyAsync(hdst[i], dout + i * m, m * sizeof(double), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess)
            st = xk::Status::Err(XK_ERR_CUDA, "device-to-host copy failed");
    if (st.ok() && cudaStreamSynchronize(s) != cudaSuccess)
        st = xk::Status::Err(XK_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    if (st.ok()) st = finish_stats(ctx, stats, used, n_good, m);
    if (!st.ok()) return fail(ctx, st);
    if (stats) {
        stats->h2d_bytes = h2d;
        stats->d2h_bytes = 4.0 * m * sizeof(double);
        stats->kernels += (n_good ? 1 : 0) + 1;
        stats->wall_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                .count();
    }
    return XK_OK;
}

}  // extern "C"
