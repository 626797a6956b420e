// Batches of independent solves: one plan for all of them, one persistent
// launch per kernel variant over every solve's items, captured once in a CUDA
// graph and replayed by xk_batch_run.
//
// The reference solves one problem per call and rebuilds its wgpu pipeline
// each time (src/gpu/kirchhoff.rs:118-241); uneven solves run back to back
// then leave most of the GPU idle whenever a solve is small. Here the items of
// all solves share one atomic work counter, so small and large solves fill the
// machine together, and the launch sequence is a graph replay.

#include <chrono>
#include <cstring>
#include <vector>

#include "xk_ctx.cuh"

struct xk_batch {
    xk_ctx* ctx = nullptr;
    int path = XK_PATH_F32PR;
    int flags = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    xk::PrWorkspace ws;
    xk::F64Workspace f64ws;
    xk::DevBuf inputs;  // device copies of host inputs and outputs
    std::vector<xk::PrSolveIn> in;
    std::vector<xk::PrPlan> plans;
    std::vector<xk_field> host_out;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double plan_ms = 0.0;
    double pairs = 0.0;
    int routed = 0;
    int kernels = 0;
    long long items = 0;
    std::string last_error;
};

namespace {

bool solve_ok(const xk_solve& s) {
    const xk_rays& r = s.rays;
    const xk_pixels& p = s.pixels;
    const xk_field& f = s.out;
    if (s.n_pix && (!p.x || !p.y || !p.z || !f.es_re || !f.es_im || !f.ep_re || !f.ep_im))
        return false;
    if (s.n_rays && (!r.x || !r.y || !r.z || !r.nx || !r.ny || !r.nz || !r.nl || !r.es_re ||
                     !r.es_im || !r.ep_re || !r.ep_im || !r.energy))
        return false;
    return true;
}

void destroy_batch(xk_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->ws.release();
    b->f64ws.rays.release();
    b->f64ws.partials.release();
    b->inputs.release();
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

// Enqueues the whole batch: the FP32-PR sweep of every planned solve, then
// the FP64 path for routed ones. Allocates nothing (the F64 workspace is
// reserved beforehand), so it can be captured.
xk::Status enqueue_batch(xk_batch* b) {
    xk::PrExecReport er;
    int kernels = 0;
    bool any_pr = false;
    for (auto& P : b->plans) any_pr |= !P.routed;
    if (any_pr) {
        XK_TRY(xk::pr_execute_enqueue(b->plans, b->ws, b->stream, b->ctx->num_sms, false, &er));
        kernels += er.kernels;
    }
    for (size_t i = 0; i < b->plans.size(); ++i) {
        if (!b->plans[i].routed) continue;
        xk::LaunchReport rep;
        const xk::PrSolveIn& s = b->in[i];
        XK_TRY(xk::f64_enqueue(s.rays, s.n, s.pix, s.m, s.out, b->f64ws, b->stream,
                               b->ctx->num_sms, &rep));
        kernels += rep.kernels;
    }
    b->kernels = kernels;
    b->items = er.n_items;
    return xk::Status::Ok();
}

xk::Status create_batch(xk_ctx* ctx, const xk_solve* solves, size_t n, int path, int flags,
                        xk_batch** out) {
    xk::NvtxRange nvtx_range("xk batch plan");
    auto t0 = std::chrono::steady_clock::now();
    xk_batch* b = new xk_batch();
    b->ctx = ctx;
    b->path = path;
    b->flags = flags;
    *out = b;
    XK_CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    XK_CUDA_TRY(cudaEventCreate(&b->ev0));
    XK_CUDA_TRY(cudaEventCreate(&b->ev1));
    // Stream-ordered allocations from the device pool: a batch created after
    // another one reuses its memory instead of mapping new memory.
    XK_TRY(xk::keep_pool_memory(ctx->device));
    b->ws.set_async(b->stream);
    b->inputs.async_stream = b->stream;
    b->f64ws.rays.async_stream = b->stream;
    b->f64ws.partials.async_stream = b->stream;
    b->f64ws.fast_reduction = ctx->f64ws.fast_reduction;
    const bool device = (flags & XK_BATCH_DEVICE) != 0;

    // Device views of every solve; host inputs are copied once into one buffer.
    b->in.resize(n);
    b->host_out.resize(n);
    size_t doubles = 0;
    if (!device)
        for (size_t i = 0; i < n; ++i) doubles += 12 * solves[i].n_rays + 7 * solves[i].n_pix;
    XK_TRY(b->inputs.ensure(std::max<size_t>(doubles, 1) * sizeof(double)));
    double* cur = b->inputs.as<double>();
    for (size_t i = 0; i < n; ++i) {
        const xk_solve& s = solves[i];
        b->pairs += (double)s.n_rays * (double)s.n_pix;
        xk::PrSolveIn& d = b->in[i];
        d.n = s.n_rays;
        d.m = s.n_pix;
        b->host_out[i] = s.out;
        if (device) {
            const xk_rays& r = s.rays;
            d.rays = xk::RaysDev{r.x, r.y, r.z, r.nx, r.ny, r.nz, r.nl,
                                 r.es_re, r.es_im, r.ep_re, r.ep_im, r.energy};
            d.pix = xk::PixDev{s.pixels.x, s.pixels.y, s.pixels.z};
            d.out = xk::FieldDev{s.out.es_re, s.out.es_im, s.out.ep_re, s.out.ep_im};
            continue;
        }
        const double* src[12] = {s.rays.x, s.rays.y, s.rays.z, s.rays.nx, s.rays.ny, s.rays.nz,
                                 s.rays.nl, s.rays.es_re, s.rays.es_im, s.rays.ep_re,
                                 s.rays.ep_im, s.rays.energy};
        const double** dst = reinterpret_cast<const double**>(&d.rays);
        for (int f = 0; f < 12; ++f) {
            dst[f] = cur;
            if (s.n_rays)
                XK_CUDA_TRY(cudaMemcpyAsync(cur, src[f], s.n_rays * sizeof(double),
                                            cudaMemcpyHostToDevice, b->stream));
            cur += s.n_rays;
        }
        const double* psrc[3] = {s.pixels.x, s.pixels.y, s.pixels.z};
        const double** pdst = reinterpret_cast<const double**>(&d.pix);
        for (int f = 0; f < 3; ++f) {
            pdst[f] = cur;
            if (s.n_pix)
                XK_CUDA_TRY(cudaMemcpyAsync(cur, psrc[f], s.n_pix * sizeof(double),
                                            cudaMemcpyHostToDevice, b->stream));
            cur += s.n_pix;
        }
        double** odst = reinterpret_cast<double**>(&d.out);
        for (int f = 0; f < 4; ++f) {
            odst[f] = cur;
            cur += s.n_pix;
        }
    }

    // One plan for every solve (FP32-PR), or all solves on the FP64 path.
    if (path == XK_PATH_F32PR) {
        int nk = 0;
        XK_TRY(xk::pr_plan(b->in.data(), (int)n, b->ws, b->stream, ctx->num_sms, ctx->pr_opts,
                           b->plans, &nk));
    } else {
        b->plans.assign(n, xk::PrPlan());
        for (auto& P : b->plans) P.routed = true;
    }
    for (size_t i = 0; i < n; ++i) {
        if (!b->plans[i].routed) continue;
        b->routed++;
        XK_TRY(xk::f64_reserve(b->in[i].n, b->in[i].m, ctx->num_sms, b->f64ws));
    }
    XK_CUDA_TRY(cudaStreamSynchronize(b->stream));
    b->plan_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    XK_TRY(xk::pr_reserve_exec(b->ws, (int)n, ctx->num_sms));
    if ((flags & XK_BATCH_NO_GRAPH) == 0) {
        XK_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        xk::Status st = enqueue_batch(b);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (!st.ok() || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();  // leave no capture error behind for later calls
            return st.ok() ? xk::Status::Err(XK_ERR_CUDA, cudaGetErrorString(e)) : st;
        }
        b->graph = g;
        XK_CUDA_TRY(cudaGraphInstantiate(&b->exec, g, 0));
    }
    return xk::Status::Ok();
}

xk::Status run_batch(xk_batch* b, xk_batch_stats* stats) {
    xk::NvtxRange nvtx_range("xk batch run");
    auto t0 = std::chrono::steady_clock::now();
    XK_CUDA_TRY(cudaEventRecord(b->ev0, b->stream));
    if (b->exec) {
        XK_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    } else {
        XK_TRY(enqueue_batch(b));
    }
    XK_CUDA_TRY(cudaEventRecord(b->ev1, b->stream));
    if ((b->flags & XK_BATCH_DEVICE) == 0) {
        for (size_t i = 0; i < b->in.size(); ++i) {
            const xk::PrSolveIn& d = b->in[i];
            if (!d.m) continue;
            const size_t bytes = d.m * sizeof(double);
            const xk_field& h = b->host_out[i];
            XK_CUDA_TRY(cudaMemcpyAsync(h.es_re, d.out.es_re, bytes, cudaMemcpyDeviceToHost, b->stream));
            XK_CUDA_TRY(cudaMemcpyAsync(h.es_im, d.out.es_im, bytes, cudaMemcpyDeviceToHost, b->stream));
            XK_CUDA_TRY(cudaMemcpyAsync(h.ep_re, d.out.ep_re, bytes, cudaMemcpyDeviceToHost, b->stream));
            XK_CUDA_TRY(cudaMemcpyAsync(h.ep_im, d.out.ep_im, bytes, cudaMemcpyDeviceToHost, b->stream));
        }
    }
    XK_CUDA_TRY(cudaStreamSynchronize(b->stream));
    bool any_pr = false;
    for (auto& P : b->plans) any_pr |= !P.routed;
    if (any_pr) {
        xk::PrExecReport er;
        XK_TRY(xk::pr_execute_finish(b->plans, b->ws, &er));
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0.f;
        XK_CUDA_TRY(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        stats->exec_ms = ms;
        stats->plan_ms = b->plan_ms;
        stats->pairs = b->pairs;
        stats->n_solves = (int)b->in.size();
        stats->routed_f64 = b->routed;
        stats->kernels = b->kernels;
        stats->n_items = b->items;
        stats->graph = b->exec ? 1 : 0;
        stats->wall_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return xk::Status::Ok();
}

}  // namespace

extern "C" {

int xk_batch_create(xk_ctx* ctx, const xk_solve* solves, size_t n, int path, int flags,
                    xk_batch** out) {
    if (!ctx || !out || (n && !solves)) return XK_ERR_INVALID;
    *out = nullptr;
    if (path != XK_PATH_F64 && path != XK_PATH_F32PR) return XK_ERR_INVALID;
    for (size_t i = 0; i < n; ++i)
        if (!solve_ok(solves[i])) {
            ctx->last_error = "batch solve " + std::to_string(i) + ": null array pointer";
            return XK_ERR_INVALID;
        }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    xk_batch* b = nullptr;
    xk::Status st = create_batch(ctx, solves, n, path, flags, &b);
    if (!st.ok()) {
        ctx->last_error = st.msg;
        destroy_batch(b);
        return st.code;
    }
    *out = b;
    return XK_OK;
}

int xk_batch_run(xk_batch* batch, xk_batch_stats* stats) {
    if (!batch) return XK_ERR_INVALID;
    std::lock_guard<std::mutex> lock(batch->ctx->mu);
    cudaSetDevice(batch->ctx->device);
    xk::Status st = run_batch(batch, stats);
    if (!st.ok()) {
        batch->ctx->last_error = st.msg;
        return st.code;
    }
    return XK_OK;
}

void xk_batch_destroy(xk_batch* batch) {
    if (!batch) return;
    std::lock_guard<std::mutex> lock(batch->ctx->mu);
    destroy_batch(batch);
}

int xk_batch_solve_plan(const xk_batch* batch, size_t i, xk_solve_plan* out) {
    if (!batch || !out || i >= batch->plans.size()) return XK_ERR_INVALID;
    const xk::PrPlan& P = batch->plans[i];
    std::memset(out, 0, sizeof(*out));
    out->path = P.routed ? XK_PATH_F64 : XK_PATH_F32PR;
    out->routed_reason = P.routed ? P.route_reason : 0;
    out->n_tiles = P.n_tiles;
    out->n_chunks = P.n_chunks;
    out->groups = P.groups;
    out->phase_bound_rad = P.phase_bound;
    out->tuned = P.tuned ? 1 : 0;
    out->sweep = P.routed ? -1 : (P.fast ? (P.lin ? 2 : 1) : 0);
    out->one_polarization = !P.routed && P.one_pol;
    return XK_OK;
}

}  // extern "C"
