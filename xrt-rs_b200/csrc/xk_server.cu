// Continuous-batching Kirchhoff server.
//
// Requests (solves of any size) arrive from any thread. Three threads serve
// them:
//   * the scheduler admits requests while the admitted set fits an HBM
//     budget and the slot count, and launches epochs: each epoch is one
//     persistent launch over work items of the planned requests — its pair
//     budget filled in order of remaining work aged by waiting time (or an
//     equal share each, as an option) — so requests that arrive while others
//     are on the GPU join the next epoch and run on the device together with
//     the older ones. Up to two epochs are queued, and epochs
//     leave a few SMs free so that planning kernels never wait behind them;
//   * the planner copies the inputs of newly admitted requests (or uses a
//     resident ray set) and plans all of them in one batched pass on a
//     high-priority stream (three host synchronisations per batch);
//   * the finisher waits for a request's final reduction, copies its field to
//     the caller's buffers, frees its memory and wakes waiters.
//
// Results are independent of the mix: a request's items accumulate into its
// own slots in a fixed order (sub-ranges of a ray group in sub order, groups
// summed in group order), whichever epoch or warp runs them.
//
// The reference has no server (one blocking call per solve,
// src/gpu/kirchhoff.rs:77-83); this is the serving layer for that call.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>
#include <vector>

#include "xk_ctx.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct RaySet {
    xk::DevBuf buf;
    size_t n = 0;
    int users = 0;
    bool released = false;
    xk::RaysDev view() const {
        const double* b = static_cast<const double*>(buf.ptr);
        return xk::RaysDev{b, b + n, b + 2 * n, b + 3 * n, b + 4 * n, b + 5 * n,
                           b + 6 * n, b + 7 * n, b + 8 * n, b + 9 * n, b + 10 * n, b + 11 * n};
    }
};

enum class ReqState { Pending, Admitted, Running, Computed, Done };

struct Req {
    uint64_t ticket = 0;
    xk_request r{};
    ReqState state = ReqState::Pending;
    int status = XK_OK;
    double bytes = 0.0;
    int path = XK_PATH_F32PR;
    bool routed = false;
    // device state
    xk::DevBuf mem;    // inputs (unless a ray set), screen points, output field
    xk::DevBuf arena;  // the plan's memory
    xk::PrPlan plan;
    xk::PrSolveIn in{};
    long long n_items = 0, next_item = 0, slice_cap = 0;
    double pairs_per_item = 0.0;
    cudaEvent_t done_ev = nullptr;
    int epochs = 0;
    Clock::time_point t_submit, t_admit, t_planned, t_done;
    RaySet* rayset = nullptr;
};

// Epochs queued on the device at once: one running and one ready keep the GPU
// busy; a third only delays new requests by one more epoch.
constexpr int kEpochRing = 2;
constexpr int kVariants = xk::kPrVariants;
constexpr int kForkStreams = 4;  // streams the kernel variants of one epoch run on
constexpr int kPlanBatch = 32;  // requests planned together at most

struct EpochSlot {
    xk::DevBuf table;     // PrSolve entries
    xk::DevBuf ctrl;      // counters + error word
    xk::PrSolve* h_table = nullptr;  // pinned
    int* h_err = nullptr;            // pinned
    cudaEvent_t ev = nullptr;
    bool in_flight = false;
    std::vector<Req*> reqs;
};

}  // namespace

struct xk_server {
    xk_ctx* ctx = nullptr;
    xk_server_opts opts{};
    xk::PrOptions pr_opts;
    int num_sms = 0;
    cudaStream_t plan_stream = nullptr, exec_stream = nullptr, io_stream = nullptr,
                 f64_stream = nullptr, out_stream = nullptr;
    // An epoch's launches of different kernel variants touch different
    // requests, so they run on parallel streams and their tails overlap.
    cudaStream_t fork_streams[kForkStreams] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kForkStreams] = {};
    std::mutex mu;
    std::condition_variable cv_work, cv_plan, cv_done;
    std::deque<Req*> pending;    // submitted, not admitted
    std::deque<Req*> to_plan;    // admitted, waiting for the planner
    std::vector<Req*> active;    // admitted, not yet computed
    std::deque<Req*> computed;   // waiting for the finisher
    std::unordered_map<uint64_t, Req*> reqs;
    std::unordered_map<uint64_t, RaySet*> raysets;
    uint64_t next_ticket = 1, next_rayset = 1;
    double used_bytes = 0.0, peak_bytes = 0.0, ray_bytes = 0.0;
    bool stopping = false, planner_done = false, worker_done = false;
    std::thread worker, planner, finisher;
    EpochSlot slots[kEpochRing];
    int next_slot = 0;
    xk::PrWorkspace plan_ws;  // planner's CUB scratch and pinned readback area
    xk::F64Workspace f64ws;
    long long alloc_count = 0;
    // statistics
    long long submitted = 0, completed = 0, failed = 0;
    std::atomic<long long> epochs{0}, kernels{0};
    double pairs_done = 0.0;
    double pairs_launched = 0.0;  // epochs launched (worker thread; read under mu)
    std::string last_error;
};

namespace {

// Device allocation that counts against the fault injector.
xk::Status checked_ensure(xk_server* s, xk::DevBuf& b, size_t bytes) {
    if (s->opts.inject_alloc_failure_every > 0) {
        long long c;
        {
            std::lock_guard<std::mutex> lock(s->mu);
            c = ++s->alloc_count;
        }
        if (c % s->opts.inject_alloc_failure_every == 0)
            return xk::Status::Err(XK_ERR_OOM, "injected allocation failure");
    }
    return b.ensure(bytes);
}

double request_bytes(const xk_server* s, const xk_request& r, size_t n_rays) {
    double b = 7.0 * 8.0 * (double)r.n_pix;                  // screen points + output
    if (r.rayset == 0) b += 12.0 * 8.0 * (double)r.n_rays;   // ray inputs
    if (r.path == XK_PATH_F32PR)
        b += (double)xk::pr_plan_bytes(n_rays, r.n_pix, s->num_sms, s->pr_opts);
    else
        b += 128.0 * (double)n_rays + 64.0 * (double)r.n_pix;  // FP64 scratch (packed rays)
    return b;
}

void finish_request(xk_server* s, Req* q, int status) {
    // Caller holds s->mu.
    q->status = status;
    q->state = ReqState::Done;
    q->t_done = Clock::now();
    if (status == XK_OK) {
        s->completed++;
        s->pairs_done += (double)q->in.n * (double)q->in.m;
    } else {
        s->failed++;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

// Caller holds s->mu: the request leaves `active` for the finisher.
void to_computed(xk_server* s, Req* q, int status) {
    if (status != XK_OK) q->status = status;
    q->state = ReqState::Computed;
    auto it = std::find(s->active.begin(), s->active.end(), q);
    if (it != s->active.end()) s->active.erase(it);
    s->computed.push_back(q);
    s->cv_work.notify_all();
}

xk::Status record_and_wait(cudaStream_t from, cudaStream_t to) {
    cudaEvent_t ev;
    XK_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e1 = cudaEventRecord(ev, from);
    cudaError_t e2 = cudaStreamWaitEvent(to, ev, 0);
    cudaEventDestroy(ev);
    XK_CUDA_TRY(e1);
    XK_CUDA_TRY(e2);
    return xk::Status::Ok();
}

// Device buffers and host-to-device copies of one request (io stream).
xk::Status copy_inputs(xk_server* s, Req* q) {
    const xk_request& r = q->r;
    const size_t n = q->rayset ? q->rayset->n : r.n_rays;
    const size_t m = r.n_pix;
    q->mem.async_stream = s->io_stream;
    const size_t doubles = (q->rayset ? 0 : 12 * n) + 7 * m;
    XK_TRY(checked_ensure(s, q->mem, std::max<size_t>(doubles, 1) * sizeof(double)));
    double* cur = q->mem.as<double>();
    if (q->rayset) {
        q->in.rays = q->rayset->view();
    } else {
        const double* src[12] = {r.rays.x, r.rays.y, r.rays.z, r.rays.nx, r.rays.ny, r.rays.nz,
                                 r.rays.nl, r.rays.es_re, r.rays.es_im, r.rays.ep_re,
                                 r.rays.ep_im, r.rays.energy};
        const double** dst = reinterpret_cast<const double**>(&q->in.rays);
        for (int f = 0; f < 12; ++f) {
            dst[f] = cur;
            if (n) XK_CUDA_TRY(cudaMemcpyAsync(cur, src[f], n * 8, cudaMemcpyHostToDevice, s->io_stream));
            cur += n;
        }
    }
    const double* psrc[3] = {r.pixels.x, r.pixels.y, r.pixels.z};
    const double** pdst = reinterpret_cast<const double**>(&q->in.pix);
    for (int f = 0; f < 3; ++f) {
        pdst[f] = cur;
        XK_CUDA_TRY(cudaMemcpyAsync(cur, psrc[f], m * 8, cudaMemcpyHostToDevice, s->io_stream));
        cur += m;
    }
    double** odst = reinterpret_cast<double**>(&q->in.out);
    for (int f = 0; f < 4; ++f) {
        odst[f] = cur;
        cur += m;
    }
    q->in.n = n;
    q->in.m = m;
    XK_CUDA_TRY(cudaEventCreateWithFlags(&q->done_ev, cudaEventDisableTiming));
    return xk::Status::Ok();
}

// The FP64 path for one request (requested, or routed by the planner).
xk::Status launch_f64(xk_server* s, Req* q) {
    q->routed = true;
    XK_TRY(record_and_wait(s->plan_stream, s->f64_stream));
    xk::LaunchReport rep;
    XK_TRY(xk::f64_enqueue(q->in.rays, q->in.n, q->in.pix, q->in.m, q->in.out, s->f64ws,
                           s->f64_stream, s->num_sms, &rep));
    s->kernels += rep.kernels;
    XK_CUDA_TRY(cudaEventRecord(q->done_ev, s->f64_stream));
    return xk::Status::Ok();
}

// Copies and plans a batch of admitted requests; runs on the planner thread.
void plan_batch(xk_server* s, std::vector<Req*>& batch) {
    xk::NvtxRange nvtx_range("xk server plan batch");
    std::vector<Req*> ok, pr;
    for (Req* q : batch) {
        xk::Status st = copy_inputs(s, q);
        std::lock_guard<std::mutex> lock(s->mu);
        if (!st.ok()) {
            s->last_error = st.msg;
            q->t_planned = Clock::now();
            to_computed(s, q, st.code);
            continue;
        }
        ok.push_back(q);
    }
    if (ok.empty()) return;
    xk::Status st = record_and_wait(s->io_stream, s->plan_stream);
    for (Req* q : ok)
        if (q->path == XK_PATH_F32PR) pr.push_back(q);
    std::vector<xk::PrPlan> plans;
    if (st.ok() && !pr.empty()) {
        std::vector<xk::PrSolveIn> in;
        std::vector<xk::DevBuf*> arenas;
        for (Req* q : pr) {
            q->arena.async_stream = s->plan_stream;
            in.push_back(q->in);
            arenas.push_back(&q->arena);
        }
        int nk = 0;
        st = xk::pr_plan(in.data(), (int)in.size(), s->plan_ws, s->plan_stream, s->num_sms,
                         s->pr_opts, plans, &nk, arenas.data());
        s->kernels += nk;
    }
    for (size_t i = 0; st.ok() && i < pr.size(); ++i) {
        Req* q = pr[i];
        q->plan = plans[i];
        xk::PrPlan& P = q->plan;
        if (P.routed) continue;
        // Slice every ray group into sub-ranges of about item_pairs pairs.
        const double rays_per_group = (double)q->in.n / P.groups;
        int subs = (int)std::ceil(rays_per_group * xk::kPrTile / s->opts.item_pairs);
        subs = std::max(1, std::min(subs, std::max(1, (int)(rays_per_group / xk::kPrStage))));
        P.dev.subs = subs;
        P.dev.n_items = (long long)P.n_tiles * P.groups * subs;
        q->n_items = P.dev.n_items;
        q->slice_cap = (long long)P.n_tiles * P.groups;
        q->pairs_per_item = rays_per_group / subs * xk::kPrTile;
        st = xk::pr_zero_partials(P, s->plan_stream);
    }
    // The execution stream must see the plans and the cleared slots before
    // the first epoch that includes these requests.
    if (st.ok()) st = record_and_wait(s->plan_stream, s->exec_stream);
    std::vector<Req*> f64;
    for (Req* q : ok)
        if (q->path == XK_PATH_F64 || q->plan.routed) f64.push_back(q);
    for (Req* q : f64) {
        if (!st.ok()) break;
        st = launch_f64(s, q);
    }
    std::lock_guard<std::mutex> lock(s->mu);
    for (Req* q : ok) {
        q->t_planned = Clock::now();
        if (!st.ok()) {
            s->last_error = st.msg;
            cudaGetLastError();
            to_computed(s, q, st.code);
        } else if (q->routed) {
            to_computed(s, q, XK_OK);
        } else {
            q->state = ReqState::Running;
        }
    }
    s->cv_work.notify_all();
}

// Waits for an epoch slot's launch, checks its error word, frees the slot.
void retire_slot(xk_server* s, EpochSlot& e) {
    if (!e.in_flight) return;
    cudaEventSynchronize(e.ev);
    e.in_flight = false;
    if (*e.h_err != 0) {
        std::lock_guard<std::mutex> lock(s->mu);
        s->last_error = "persistent kernel: a bounded wait for a ray stage ran out";
        for (Req* q : e.reqs)
            if (q->state != ReqState::Done) q->status = XK_ERR_TIMEOUT;
    }
    e.reqs.clear();
}

// Builds and launches one epoch over the planned FP32-PR requests.
xk::Status run_epoch(xk_server* s, std::vector<Req*>& runnable) {
    xk::NvtxRange nvtx_range("xk server epoch");
    EpochSlot& e = s->slots[s->next_slot];
    s->next_slot = (s->next_slot + 1) % kEpochRing;
    retire_slot(s, e);

    struct Take {
        Req* q;
        long long first, count;
    };
    std::vector<Take> takes;
    auto take = [&](Req* q, double pairs) {
        long long quota = (long long)std::max(1.0, std::floor(pairs / std::max(1.0, q->pairs_per_item)));
        quota = std::min(quota, q->slice_cap);
        quota = std::min(quota, q->n_items - q->next_item);
        if (quota <= 0) return 0.0;
        takes.push_back({q, q->next_item, quota});
        return (double)quota * q->pairs_per_item;
    };
    if (s->opts.policy == XK_SERVE_EQUAL_SHARE) {
        // Every running request gets the same share of the epoch's pairs.
        const double share = s->opts.epoch_pairs / std::max<size_t>(1, runnable.size());
        for (Req* q : runnable) take(q, share);
    } else {
        // Shortest remaining work first, aged: the epoch's pairs go to the
        // requests in order of remaining pairs / (1 + waited / aging_ms).
        // Small requests leave in few epochs; a large one's key shrinks as it
        // waits (half after aging_ms, a third after twice that), so it is not
        // starved.
        const Clock::time_point now = Clock::now();
        std::vector<std::pair<double, Req*>> order;
        order.reserve(runnable.size());
        for (Req* q : runnable) {
            const double left = (double)(q->n_items - q->next_item) * q->pairs_per_item;
            const double waited = ms_between(q->t_submit, now);
            order.push_back({left / (1.0 + waited / s->opts.aging_ms), q});
        }
        std::stable_sort(order.begin(), order.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
        double budget = s->opts.epoch_pairs;
        for (const auto& o : order) {
            if (budget <= 0.0) break;
            budget -= take(o.second, budget);
        }
    }
    if (takes.empty()) return xk::Status::Ok();

    // One table, grouped by kernel variant.
    int tab = 0;
    long long counts[kVariants] = {};
    int first[kVariants] = {}, nsol[kVariants] = {};
    for (int v = 0; v < kVariants; ++v) {
        first[v] = tab;
        for (const Take& t : takes) {
            const xk::PrPlan& P = t.q->plan;
            if (P.variant() != v) continue;
            xk::PrSolve d = P.dev;
            d.item_begin = counts[v];
            d.item_offset = t.first;
            e.h_table[tab++] = d;
            counts[v] += t.count;
            nsol[v]++;
        }
    }
    XK_CUDA_TRY(cudaMemcpyAsync(e.table.ptr, e.h_table, tab * sizeof(xk::PrSolve),
                                cudaMemcpyHostToDevice, s->exec_stream));
    XK_CUDA_TRY(cudaMemsetAsync(e.ctrl.ptr, 0, xk::kPrCtrlBytes, s->exec_stream));
    unsigned long long* counters = e.ctrl.as<unsigned long long>();
    int* d_err = reinterpret_cast<int*>(e.ctrl.as<char>() + xk::kPrCtrlErrOffset);
    const int sms = std::max(1, s->num_sms - std::max(0, s->opts.reserve_sms));
    XK_CUDA_TRY(cudaEventRecord(s->fork_ev, s->exec_stream));
    int forks = 0;
    for (int v = 0; v < kVariants; ++v) {
        if (!nsol[v]) continue;
        cudaStream_t st = s->fork_streams[forks % kForkStreams];
        if (forks < kForkStreams) XK_CUDA_TRY(cudaStreamWaitEvent(st, s->fork_ev, 0));
        XK_TRY(xk::pr_launch(e.table.as<xk::PrSolve>() + first[v], nsol[v], counts[v], v,
                             counters + v, d_err, st, sms, 0));
        s->kernels++;
        ++forks;
    }
    for (int f = 0; f < std::min(forks, kForkStreams); ++f) {
        XK_CUDA_TRY(cudaEventRecord(s->join_ev[f], s->fork_streams[f]));
        XK_CUDA_TRY(cudaStreamWaitEvent(s->exec_stream, s->join_ev[f], 0));
    }
    XK_CUDA_TRY(cudaMemcpyAsync(e.h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s->exec_stream));
    double launched = 0.0;
    for (const Take& t : takes) launched += (double)t.count * t.q->pairs_per_item;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->pairs_launched += launched;
    }
    for (const Take& t : takes) {
        t.q->next_item += t.count;
        t.q->epochs++;
        e.reqs.push_back(t.q);
        if (t.q->next_item >= t.q->n_items) {
            XK_TRY(xk::pr_finalize(t.q->plan, s->exec_stream));
            s->kernels++;
            XK_CUDA_TRY(cudaEventRecord(t.q->done_ev, s->exec_stream));
        }
    }
    XK_CUDA_TRY(cudaEventRecord(e.ev, s->exec_stream));
    e.in_flight = true;
    s->epochs++;
    return xk::Status::Ok();
}

void release_request_memory(xk_server* s, Req* q) {
    q->arena.release();
    q->mem.release();
    if (q->done_ev) cudaEventDestroy(q->done_ev);
    q->done_ev = nullptr;
    std::lock_guard<std::mutex> lock(s->mu);
    s->used_bytes -= q->bytes;
    if (q->rayset) {
        q->rayset->users--;
        if (q->rayset->released && q->rayset->users == 0) {
            s->ray_bytes -= 96.0 * q->rayset->n;
            s->used_bytes -= 96.0 * q->rayset->n;
            q->rayset->buf.release();
            delete q->rayset;
        }
        q->rayset = nullptr;
    }
}

void planner_loop(xk_server* s) {
    cudaSetDevice(s->ctx->device);
    while (true) {
        std::vector<Req*> batch;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv_plan.wait_for(lock, std::chrono::milliseconds(5),
                                [&] { return !s->to_plan.empty() || s->stopping; });
            if (s->stopping) break;
            while (!s->to_plan.empty() && (int)batch.size() < kPlanBatch) {
                batch.push_back(s->to_plan.front());
                s->to_plan.pop_front();
            }
        }
        if (!batch.empty()) plan_batch(s, batch);
    }
    std::lock_guard<std::mutex> lock(s->mu);
    s->planner_done = true;
    s->cv_work.notify_all();
}

void worker_loop(xk_server* s) {
    cudaSetDevice(s->ctx->device);
    while (true) {
        std::vector<Req*> runnable;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            auto can_admit = [&] {
                if (s->pending.empty() || (int)s->active.size() >= s->opts.max_active) return false;
                const double b = s->pending.front()->bytes;
                return s->active.empty() || b > s->opts.hbm_budget_bytes ||
                       s->used_bytes + b <= s->opts.hbm_budget_bytes;
            };
            auto has_work = [&] {
                if (s->stopping) return true;
                if (can_admit()) return true;
                for (Req* q : s->active)
                    if (q->state == ReqState::Running && q->next_item < q->n_items) return true;
                return false;
            };
            if (!has_work()) s->cv_work.wait_for(lock, std::chrono::milliseconds(2), has_work);
            if (s->stopping) {
                // Wait for the planner to stop and for the launched epochs to
                // finish (no kernel may touch memory that is about to be
                // freed), then cancel everything not yet completed.
                s->cv_work.wait(lock, [&] { return s->planner_done; });
                lock.unlock();
                for (EpochSlot& e : s->slots) retire_slot(s, e);
                lock.lock();
                while (!s->pending.empty()) {
                    Req* q = s->pending.front();
                    s->pending.pop_front();
                    finish_request(s, q, XK_ERR_SHUTDOWN);
                }
                while (!s->to_plan.empty()) {
                    Req* q = s->to_plan.front();
                    s->to_plan.pop_front();
                    auto it = std::find(s->active.begin(), s->active.end(), q);
                    if (it != s->active.end()) s->active.erase(it);
                    s->used_bytes -= q->bytes;
                    finish_request(s, q, XK_ERR_SHUTDOWN);
                }
                for (Req* q : std::vector<Req*>(s->active)) to_computed(s, q, XK_ERR_SHUTDOWN);
                s->worker_done = true;
                s->cv_work.notify_all();
                break;
            }
            // Admission: FIFO while the budget and the slot count allow.
            while (can_admit()) {
                Req* q = s->pending.front();
                s->pending.pop_front();
                if (q->bytes > s->opts.hbm_budget_bytes) {
                    finish_request(s, q, XK_ERR_BUDGET);
                    continue;
                }
                s->used_bytes += q->bytes;
                s->peak_bytes = std::max(s->peak_bytes, s->used_bytes);
                q->state = ReqState::Admitted;
                q->t_admit = Clock::now();
                s->active.push_back(q);
                s->to_plan.push_back(q);
                s->cv_plan.notify_all();
            }
            for (Req* q : s->active)
                if (q->state == ReqState::Running && q->next_item < q->n_items) runnable.push_back(q);
        }
        if (runnable.empty()) continue;
        xk::Status st = run_epoch(s, runnable);
        if (!st.ok()) {
            // Requests leave with an error: let launched epochs finish first.
            cudaGetLastError();
            for (EpochSlot& e : s->slots) retire_slot(s, e);
        }
        std::lock_guard<std::mutex> lock(s->mu);
        if (!st.ok()) s->last_error = st.msg;
        for (Req* q : runnable)
            if (q->next_item >= q->n_items || !st.ok()) to_computed(s, q, st.ok() ? XK_OK : st.code);
    }
}

void finisher_loop(xk_server* s) {
    cudaSetDevice(s->ctx->device);
    while (true) {
        Req* q = nullptr;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv_work.wait_for(lock, std::chrono::milliseconds(2),
                                [&] { return !s->computed.empty() || s->worker_done; });
            if (s->computed.empty()) {
                if (s->worker_done) break;
                continue;
            }
            q = s->computed.front();
            s->computed.pop_front();
        }
        xk::NvtxRange nvtx_range("xk server finish request");
        int status = q->status;
        if (q->done_ev) {
            cudaError_t e = cudaEventSynchronize(q->done_ev);
            if (e != cudaSuccess && status == XK_OK) status = XK_ERR_CUDA;
        }
        if (status == XK_OK && q->in.m) {
            const size_t bytes = q->in.m * sizeof(double);
            const xk_field& h = q->r.out;
            double* dst[4] = {h.es_re, h.es_im, h.ep_re, h.ep_im};
            const double* src[4] = {q->in.out.es_re, q->in.out.es_im, q->in.out.ep_re, q->in.out.ep_im};
            for (int f = 0; f < 4; ++f)
                if (cudaMemcpyAsync(dst[f], src[f], bytes, cudaMemcpyDeviceToHost, s->out_stream) != cudaSuccess)
                    status = XK_ERR_CUDA;
            if (cudaStreamSynchronize(s->out_stream) != cudaSuccess) status = XK_ERR_CUDA;
        }
        if (status != XK_OK) {
            // A failed request may still have planning or FP64 work queued on
            // its memory: let it drain before the memory is freed.
            cudaStreamSynchronize(s->plan_stream);
            cudaStreamSynchronize(s->f64_stream);
            cudaGetLastError();
        }
        release_request_memory(s, q);
        std::lock_guard<std::mutex> lock(s->mu);
        finish_request(s, q, status);
    }
}

void destroy_server(xk_server* s) {
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
        if (!s->planner.joinable()) s->planner_done = true;
        if (!s->worker.joinable()) s->worker_done = true;
    }
    s->cv_work.notify_all();
    s->cv_plan.notify_all();
    if (s->planner.joinable()) s->planner.join();
    if (s->worker.joinable()) s->worker.join();
    if (s->finisher.joinable()) s->finisher.join();
    cudaSetDevice(s->ctx->device);
    for (EpochSlot& e : s->slots) {
        e.table.release();
        e.ctrl.release();
        if (e.ev) cudaEventDestroy(e.ev);
        if (e.h_table) cudaFreeHost(e.h_table);
        if (e.h_err) cudaFreeHost(e.h_err);
    }
    for (auto& kv : s->reqs) {
        Req* q = kv.second;
        q->arena.release();
        q->mem.release();
        if (q->done_ev) cudaEventDestroy(q->done_ev);
        delete q;
    }
    for (auto& kv : s->raysets) {
        kv.second->buf.release();
        delete kv.second;
    }
    s->plan_ws.release();
    s->f64ws.rays.release();
    s->f64ws.partials.release();
    for (int f = 0; f < kForkStreams; ++f) {
        if (s->fork_streams[f]) {
            cudaStreamSynchronize(s->fork_streams[f]);
            cudaStreamDestroy(s->fork_streams[f]);
        }
        if (s->join_ev[f]) cudaEventDestroy(s->join_ev[f]);
    }
    if (s->fork_ev) cudaEventDestroy(s->fork_ev);
    for (cudaStream_t st : {s->plan_stream, s->exec_stream, s->io_stream, s->f64_stream, s->out_stream})
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    delete s;
}

xk::Status create_server(xk_ctx* ctx, const xk_server_opts* opts, xk_server** out) {
    xk_server* s = new xk_server();
    *out = s;
    s->ctx = ctx;
    s->num_sms = ctx->num_sms;
    if (opts) s->opts = *opts;
    if (s->opts.hbm_budget_bytes <= 0) s->opts.hbm_budget_bytes = 120e9;
    if (s->opts.epoch_pairs <= 0) s->opts.epoch_pairs = 3e10;
    if (s->opts.max_active <= 0) s->opts.max_active = 64;
    if (s->opts.item_pairs <= 0) s->opts.item_pairs = 1e6;
    if (s->opts.reserve_sms <= 0) s->opts.reserve_sms = 8;
    if (s->opts.policy != XK_SERVE_SHORTEST_AGED && s->opts.policy != XK_SERVE_EQUAL_SHARE)
        return xk::Status::Err(XK_ERR_INVALID, "unknown serving policy");
    if (s->opts.aging_ms <= 0) s->opts.aging_ms = 1000.0;
    s->opts.reserve_sms = std::min(s->opts.reserve_sms, s->num_sms - 1);
    s->pr_opts = ctx->pr_opts;
    // Keep freed stream-ordered memory in the pool instead of returning it to
    // the driver at every synchronisation.
    XK_TRY(xk::keep_pool_memory(ctx->device));
    int lo = 0, hi = 0;
    XK_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    XK_CUDA_TRY(cudaStreamCreateWithPriority(&s->plan_stream, cudaStreamNonBlocking, hi));
    XK_CUDA_TRY(cudaStreamCreateWithPriority(&s->exec_stream, cudaStreamNonBlocking, lo));
    XK_CUDA_TRY(cudaStreamCreateWithPriority(&s->io_stream, cudaStreamNonBlocking, hi));
    XK_CUDA_TRY(cudaStreamCreateWithPriority(&s->f64_stream, cudaStreamNonBlocking, lo));
    XK_CUDA_TRY(cudaStreamCreateWithPriority(&s->out_stream, cudaStreamNonBlocking, hi));
    for (int f = 0; f < kForkStreams; ++f) {
        XK_CUDA_TRY(cudaStreamCreateWithPriority(&s->fork_streams[f], cudaStreamNonBlocking, lo));
        XK_CUDA_TRY(cudaEventCreateWithFlags(&s->join_ev[f], cudaEventDisableTiming));
    }
    XK_CUDA_TRY(cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming));
    for (EpochSlot& e : s->slots) {
        XK_TRY(e.table.ensure(kVariants * (size_t)std::max(1, s->opts.max_active) * sizeof(xk::PrSolve)));
        XK_TRY(e.ctrl.ensure(xk::kPrCtrlBytes));
        XK_CUDA_TRY(cudaMallocHost(&e.h_table,
                                   kVariants * (size_t)std::max(1, s->opts.max_active) * sizeof(xk::PrSolve)));
        XK_CUDA_TRY(cudaMallocHost(&e.h_err, 64));
        *e.h_err = 0;
        XK_CUDA_TRY(cudaEventCreateWithFlags(&e.ev, cudaEventDisableTiming));
    }
    // The planner's scratch: CUB temporaries grow stream-ordered; the pinned
    // readback area is sized once for the largest planning batch.
    s->plan_ws.set_async(s->plan_stream);
    XK_TRY(xk::pr_reserve_plan_host(s->plan_ws, kPlanBatch, s->num_sms));
    s->f64ws.rays.async_stream = s->f64_stream;
    s->f64ws.partials.async_stream = s->f64_stream;
    s->f64ws.fast_reduction = ctx->f64ws.fast_reduction;
    s->worker = std::thread(worker_loop, s);
    s->planner = std::thread(planner_loop, s);
    s->finisher = std::thread(finisher_loop, s);
    return xk::Status::Ok();
}

}  // namespace

extern "C" {

int xk_server_create(xk_ctx* ctx, const xk_server_opts* opts, xk_server** out) {
    if (!ctx || !out) return XK_ERR_INVALID;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    xk_server* s = nullptr;
    xk::Status st = create_server(ctx, opts, &s);
    if (!st.ok()) {
        ctx->last_error = st.msg;
        if (s) destroy_server(s);
        return st.code;
    }
    *out = s;
    return XK_OK;
}

void xk_server_destroy(xk_server* server) {
    if (server) destroy_server(server);
}

int xk_server_upload_rays(xk_server* s, const xk_rays* rays, size_t n, uint64_t* handle) {
    if (!s || !rays || !handle || n == 0) return XK_ERR_INVALID;
    if (!rays->x || !rays->y || !rays->z || !rays->nx || !rays->ny || !rays->nz || !rays->nl ||
        !rays->es_re || !rays->es_im || !rays->ep_re || !rays->ep_im || !rays->energy)
        return XK_ERR_INVALID;
    const double bytes = 96.0 * (double)n;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->used_bytes + bytes > s->opts.hbm_budget_bytes) return XK_ERR_BUDGET;
        s->used_bytes += bytes;
        s->ray_bytes += bytes;
        s->peak_bytes = std::max(s->peak_bytes, s->used_bytes);
    }
    cudaSetDevice(s->ctx->device);
    RaySet* rs = new RaySet();
    rs->n = n;
    rs->buf.async_stream = s->io_stream;
    const double* src[12] = {rays->x, rays->y, rays->z, rays->nx, rays->ny, rays->nz, rays->nl,
                             rays->es_re, rays->es_im, rays->ep_re, rays->ep_im, rays->energy};
    int rc = XK_OK;
    cudaStream_t st = s->io_stream;
    if (!rs->buf.ensure(12 * n * sizeof(double)).ok()) rc = XK_ERR_OOM;
    for (int f = 0; f < 12 && rc == XK_OK; ++f)
        if (cudaMemcpyAsync(rs->buf.as<double>() + f * n, src[f], n * 8, cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
            rc = XK_ERR_CUDA;
    // Requests that use the set are planned on other streams: the set must be
    // complete before this call returns.
    if (cudaStreamSynchronize(st) != cudaSuccess && rc == XK_OK) rc = XK_ERR_CUDA;
    std::lock_guard<std::mutex> lock(s->mu);
    if (rc != XK_OK) {
        s->used_bytes -= bytes;
        s->ray_bytes -= bytes;
        rs->buf.release();
        delete rs;
        return rc;
    }
    *handle = s->next_rayset++;
    s->raysets[*handle] = rs;
    return XK_OK;
}

int xk_server_upload_beam(xk_server* s, const xk_beam* beam, size_t n_beam,
                          const double* normals, const size_t* good, size_t n_good,
                          uint64_t* handle) {
    if (!s || !beam || !normals || !good || !handle || n_good == 0) return XK_ERR_INVALID;
    if (!beam->x || !beam->y || !beam->z || !beam->a || !beam->b || !beam->c || !beam->e)
        return XK_ERR_INVALID;
    const int amps = !!beam->es_re + !!beam->es_im + !!beam->ep_re + !!beam->ep_im;
    if (amps != 0 && amps != 4) return XK_ERR_INVALID;
    // beam_to_diffraction_rays indexes the beam with `good` (the reference
    // panics on an index out of range).
    for (size_t i = 0; i < n_good; ++i)
        if (good[i] >= n_beam) return XK_ERR_INVALID;
    static_assert(sizeof(size_t) == sizeof(uint64_t), "good indices are copied as 64-bit words");
    const double bytes = 96.0 * (double)n_good;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->used_bytes + bytes > s->opts.hbm_budget_bytes) return XK_ERR_BUDGET;
        s->used_bytes += bytes;
        s->ray_bytes += bytes;
        s->peak_bytes = std::max(s->peak_bytes, s->used_bytes);
    }
    cudaSetDevice(s->ctx->device);
    RaySet* rs = new RaySet();
    rs->n = n_good;
    cudaStream_t st = s->io_stream;
    rs->buf.async_stream = st;
    // The beam's columns, normals and indices are staged in a transient
    // stream-ordered allocation, gathered into the set's 12 columns by
    // beam_rays_kernel (xk_wave.cu) and freed before the call returns.
    xk::DevBuf stage;
    stage.async_stream = st;
    const int cols = amps ? 11 : 7;
    const size_t nb = n_beam * sizeof(double);
    xk::Status stt = rs->buf.ensure(12 * n_good * sizeof(double));
    if (stt.ok()) stt = stage.ensure((size_t)(cols + 3) * nb + n_good * sizeof(uint64_t));
    xk::BeamDev bd{};
    const uint64_t* d_good = nullptr;
    if (stt.ok()) {
        const double* src[11] = {beam->x, beam->y, beam->z, beam->a, beam->b, beam->c, beam->e,
                                 beam->es_re, beam->es_im, beam->ep_re, beam->ep_im};
        const double** dst = reinterpret_cast<const double**>(&bd);
        double* d = stage.as<double>();
        for (int f = 0; f < cols && stt.ok(); ++f, d += n_beam) {
            dst[f] = d;
            stt = xk::Status::FromCuda(cudaMemcpyAsync(d, src[f], nb, cudaMemcpyHostToDevice, st));
        }
        bd.normals = d;
        if (stt.ok())
            stt = xk::Status::FromCuda(
                cudaMemcpyAsync(d, normals, 3 * nb, cudaMemcpyHostToDevice, st));
        d_good = reinterpret_cast<const uint64_t*>(d + 3 * n_beam);
        if (stt.ok())
            stt = xk::Status::FromCuda(cudaMemcpyAsync(const_cast<uint64_t*>(d_good), good,
                                                       n_good * sizeof(uint64_t),
                                                       cudaMemcpyHostToDevice, st));
    }
    if (stt.ok()) {
        double* out[12];
        for (int f = 0; f < 12; ++f) out[f] = rs->buf.as<double>() + (size_t)f * n_good;
        stt = xk::beam_rays_enqueue(bd, d_good, n_good, out, st);
    }
    stage.release();
    // Requests that use the set are planned on other streams: the set must be
    // complete before this call returns.
    const cudaError_t se = cudaStreamSynchronize(st);
    if (stt.ok() && se != cudaSuccess) stt = xk::Status::FromCuda(se);
    std::lock_guard<std::mutex> lock(s->mu);
    if (!stt.ok()) {
        s->used_bytes -= bytes;
        s->ray_bytes -= bytes;
        rs->buf.release();
        delete rs;
        return stt.code;
    }
    *handle = s->next_rayset++;
    s->raysets[*handle] = rs;
    return XK_OK;
}

int xk_server_release_rays(xk_server* s, uint64_t handle) {
    if (!s) return XK_ERR_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->raysets.find(handle);
    if (it == s->raysets.end()) return XK_ERR_NOT_FOUND;
    RaySet* rs = it->second;
    s->raysets.erase(it);
    rs->released = true;
    if (rs->users == 0) {
        s->ray_bytes -= 96.0 * rs->n;
        s->used_bytes -= 96.0 * rs->n;
        rs->buf.release();
        delete rs;
    }
    return XK_OK;
}

int xk_server_submit(xk_server* s, const xk_request* req, uint64_t* ticket) {
    if (!s || !req || !ticket) return XK_ERR_INVALID;
    if (req->path != XK_PATH_F64 && req->path != XK_PATH_F32PR) return XK_ERR_INVALID;
    const xk_pixels& p = req->pixels;
    const xk_field& f = req->out;
    if (req->n_pix == 0 || !p.x || !p.y || !p.z || !f.es_re || !f.es_im || !f.ep_re || !f.ep_im)
        return XK_ERR_INVALID;
    Req* q = new Req();
    q->r = *req;
    q->path = req->path;
    q->t_submit = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    size_t n = req->n_rays;
    if (req->rayset) {
        auto it = s->raysets.find(req->rayset);
        if (it == s->raysets.end()) {
            delete q;
            return XK_ERR_NOT_FOUND;
        }
        q->rayset = it->second;
        q->rayset->users++;
        n = q->rayset->n;
    } else if (n && (!req->rays.x || !req->rays.y || !req->rays.z || !req->rays.nx ||
                     !req->rays.ny || !req->rays.nz || !req->rays.nl || !req->rays.es_re ||
                     !req->rays.es_im || !req->rays.ep_re || !req->rays.ep_im ||
                     !req->rays.energy)) {
        delete q;
        return XK_ERR_INVALID;
    }
    if (s->stopping) {
        if (q->rayset) q->rayset->users--;
        delete q;
        return XK_ERR_SHUTDOWN;
    }
    q->bytes = request_bytes(s, *req, n);
    q->ticket = s->next_ticket++;
    s->reqs[q->ticket] = q;
    s->pending.push_back(q);
    s->submitted++;
    *ticket = q->ticket;
    s->cv_work.notify_all();
    return XK_OK;
}

int xk_server_wait(xk_server* s, uint64_t ticket, double timeout_ms, xk_request_stats* stats) {
    if (!s) return XK_ERR_INVALID;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return XK_ERR_NOT_FOUND;
    Req* q = it->second;
    auto done = [&] { return q->state == ReqState::Done; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lock, done);
    } else if (!s->cv_done.wait_for(lock, std::chrono::duration<double, std::milli>(timeout_ms), done)) {
        return XK_ERR_TIMEOUT;
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->pairs = (double)q->in.n * (double)q->in.m;
        stats->status = q->status;
        stats->path = q->routed ? XK_PATH_F64 : XK_PATH_F32PR;
        stats->epochs = q->epochs;
        if (q->t_admit.time_since_epoch().count()) {
            stats->queue_ms = ms_between(q->t_submit, q->t_admit);
            stats->plan_ms = ms_between(q->t_admit, q->t_planned);
            stats->run_ms = ms_between(q->t_planned, q->t_done);
        }
        stats->total_ms = ms_between(q->t_submit, q->t_done);
    }
    const int status = q->status;
    s->reqs.erase(it);
    delete q;
    return status;
}

int xk_server_get_stats(xk_server* s, xk_server_stats* out) {
    if (!s || !out) return XK_ERR_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->epochs = s->epochs.load();
    out->kernels = s->kernels.load();
    out->pending = (long long)s->pending.size();
    out->active = (long long)s->active.size();
    out->pairs_done = s->pairs_done;
    out->pairs_launched = s->pairs_launched;
    out->used_bytes = s->used_bytes;
    out->peak_bytes = s->peak_bytes;
    out->resident_ray_bytes = s->ray_bytes;
    return XK_OK;
}

}  // extern "C"
