// FP32 phase-reduced Kirchhoff path: planner + persistent kernel.
#pragma once

#include <map>
#include <mutex>
#include <vector>

#include "xk_internal.cuh"

namespace xk {

// Geometry of the work decomposition.
constexpr int kPrWarpsPerCta = 4;
constexpr int kPrStage = 56;          // rays per shared-memory stage
constexpr int kPrPpl = 8;             // screen points per lane
constexpr int kPrTile = 32 * kPrPpl;  // screen points per tile (one warp)

// Settings the autotuner found best for one class of solves.
struct PrTuned {
    double phase_budget = 512.0;
    long long items_per_warp = 16;
    int sweep = -1;
};

// Autotuned settings per bucket of solves: (energy, distance, ray count,
// screen-point count), each on a log2 scale (energy in eV and distance in mm
// rounded to the nearest power of two, counts by their leading power of
// two). The ray-group count is fixed before the planner knows energy and
// distance, so items per warp is also kept per (ray count, screen count).
struct PrTuneCache {
    std::mutex mu;
    std::map<uint64_t, PrTuned> full;
    std::map<uint32_t, long long> ipw;
    bool use = true;  // apply cached settings to matching solves
    static uint32_t size_key(size_t n, size_t m);
    static uint64_t full_key(double energy_ev, double dist_mm, size_t n, size_t m);
    void store(double energy_ev, double dist_mm, size_t n, size_t m, const PrTuned& t);
    bool find(double energy_ev, double dist_mm, size_t n, size_t m, PrTuned* t);
    bool find_ipw(size_t n, size_t m, long long* ipw_out);
    size_t size();
    void clear();
};

// Planner knobs.
struct PrOptions {
    double phase_budget = 512.0;  // cap on |FP32 residual phase| [rad]
    // Requested relative L2 error of the field; the planner derives the
    // residual-phase budget from it (effective_phase_budget).
    double tolerance = 1e-4;
    int groups = 0;               // ray groups per tile; 0 = automatic
    int sweep = -1;               // -1 automatic, 0 SFU reciprocal, 1 packed + quadratic
                                  // series reciprocal, 2 packed + linear series
    long long items_per_warp = 16;  // target items per resident warp (automatic groups)
    int polarization = -1;        // -1 automatic, 0 always sum Es and Ep separately
    PrTuneCache* tune = nullptr;  // per-bucket settings that override the above, or null
};

// Launch controls of the persistent kernel: the poll limit of every bounded
// wait, and a test hook that arms the first ray stage of item 0 with
// `stall_bytes` more than its bulk copy delivers, so that stage's barrier
// never completes and the wait runs out (the copy itself lands; nothing is
// left in flight). 0 in production.
struct PrCtl {
    uint32_t wait_limit = 1u << 24;
    uint32_t stall_bytes = 0;
};

// Residual-phase budget [rad] per unit of requested relative error. The
// FP32 residual phase carries rounding errors proportional to its size (its
// own rounding, that of the terms it is formed from and of the sin/cos
// argument): on the worst fields measured — two equal rays in phase at 1 keV
// and 100 mm, whose pairs all sit near the bound — the field error was
// 1.45e-7 per rad of budget. The constant keeps that worst case at 0.4 of the
// requested tolerance.
constexpr double kPhasePerTolerance = 2.75e6;

// The budget the planner sizes ray chunks for: the tolerance's, capped by
// `phase_budget`.
inline double effective_phase_budget(const PrOptions& o) {
    const double t = o.tolerance * kPhasePerTolerance;
    return t < o.phase_budget ? t : o.phase_budget;
}

// Reasons a solve is routed to the FP64 path (xk_route_reason).
constexpr int kRouteReasonCount = 9;
extern const char* const kRouteReasons[kRouteReasonCount];

// Sorted ray record as the planner writes it and TMA stages it: position
// relative to its chunk centre in FP64, amplitudes, normal and obliquity in
// FP32. 64 bytes, 16-byte aligned.
struct __align__(16) PrRawRay {
    double rx, ry, rz;
    float es_re, es_im, ep_re, ep_im;
    float nx, ny, nz, nl;
    float pad0, pad1;
};
static_assert(sizeof(PrRawRay) == 64, "record is 64 bytes");

// Device-side description of one planned solve (read by the persistent
// kernel).
struct PrSolve {
    const PrRawRay* recs;         // [n_rays] in chunk order
    const int* chunk_begin;       // [n_chunks + 1]
    const double* chunk_center;   // [3 * n_chunks]
    const int* n_chunks_dev;      // scalar
    const double *tpx, *tpy, *tpz;  // screen points in tile-slot order (padding = tile centre)
    const double* tile_center;    // [3 * n_tiles]
    const int* group_order;       // [groups] ray groups by decreasing estimated cost
    double* partial;              // [groups][4][n_tiles * kPrTile], tile-slot order
    long long item_begin;         // first global item of this solve in its launch
    long long item_offset;        // first of the solve's own items covered by the launch
    long long n_items;            // n_tiles * groups * subs
    int n_rays, n_tiles, groups;
    int subs;                     // sub-ranges per ray group (items per (group, tile))
    double k;                     // wavenumber [1/mm]
    double kt;                    // k / (2 pi), high part
    double kt_lo;                 // k / (2 pi), low part (double-double)
    float unx, uny, unz;          // the common normal (uniform-normal kernels)
    int amp_src;                  // one-polarization kernels: 0 sum es, 1 sum ep
};

// One solve's inputs (device pointers).
struct PrSolveIn {
    RaysDev rays;
    size_t n;
    PixDev pix;
    size_t m;
    FieldDev out;
};

// Host-side result of planning one solve.
struct PrPlan {
    bool routed = false;
    int route_reason = 0;
    bool uniform_normal = false;
    bool fast = false;  // packed sweep with Newton reciprocal
    bool fold = false;  // base phase folded into the per-pair phase (near field)
    bool lin = false;   // packed sweep with the series reciprocal cut after the linear term
    // Every ray's (es, ep) is a multiple of one complex pair: the kernel sums
    // A = sum a_j U_j for one amplitude column and the field is
    // (Es, Ep) = (pol_es, pol_ep) * A.
    bool one_pol = false;
    double pol_es[2] = {1.0, 0.0}, pol_ep[2] = {0.0, 0.0};
    // Kernel variant: bit 0 uniform normal, bit 1 packed sweep, bit 2 folded,
    // bit 3 one polarization, bit 4 linear series (packed sweep only).
    int variant() const {
        return (uniform_normal ? 1 : 0) | (fast ? 2 : 0) | (fold ? 4 : 0) | (one_pol ? 8 : 0) |
               (fast && lin ? 16 : 0);
    }
    int n_tiles = 0, groups = 0, n_chunks = 0;
    double phase_bound = 0.0, rcp_bound = 0.0;
    double energy_ev = 0.0, dist_mm = 0.0;  // the solve's energy and ray/screen box distance
    bool tuned = false;                     // settings came from the tuning cache
    PrSolve dev{};
    const int* tile_perm = nullptr;  // slot -> original screen point, -1 = padding
    int m = 0;
    FieldDev out{};
    int* n_chunks_host = nullptr;    // filled after execution
};

struct PrExecReport {
    int kernels = 0;
    float main_kernel_ms = 0.f;
    long long n_items = 0;
};

struct PrWorkspace {
    DevBuf arena;
    DevBuf cub_tmp;
    DevBuf solves;  // PrSolve tables for the persistent launches
    DevBuf ctrl;    // item counters + error flag
    cudaEvent_t ev[2] = {nullptr, nullptr};  // bracket the pair kernels
    void* host = nullptr;  // pinned readback / upload area
    size_t host_bytes = 0;
    int* host_err = nullptr;  // error word copied back by the last execution
    bool host_borrowed = false;  // `host` belongs to the caller: never freed here
    PrCtl ctl;                   // wait limit; stall_bytes is cleared after one execution
    Status ensure_host(size_t bytes);
    void release();
    // Stream-ordered allocation for every device buffer of this workspace.
    void set_async(cudaStream_t s) {
        arena.async_stream = cub_tmp.async_stream = solves.async_stream = ctrl.async_stream = s;
    }
};

// Bytes of device memory pr_plan needs for one solve of n rays and m screen
// points (arena and CUB scratch), for admission control.
size_t pr_plan_bytes(size_t n, size_t m, int num_sms, const PrOptions& opt);

// Plans `count` solves in one pass (three host synchronisations for the
// whole batch). Plans reference memory in ws.arena until the next call, or,
// with `arenas`, solve s's memory in *arenas[s] (grown as needed), so that
// solves planned together can be released one by one.
Status pr_plan(const PrSolveIn* in, int count, PrWorkspace& ws, cudaStream_t stream, int num_sms,
               const PrOptions& opt, std::vector<PrPlan>& plans, int* kernels,
               DevBuf* const* arenas = nullptr);

// Allocates everything pr_execute_enqueue needs for `count` solves, so that a
// following enqueue allocates nothing (required while capturing a graph).
// Pinned readback area for planning up to `count` solves at once (so that a
// long-lived planner never reallocates it).
Status pr_reserve_plan_host(PrWorkspace& ws, int count, int num_sms);
Status pr_reserve_exec(PrWorkspace& ws, int count, int num_sms);

// Enqueues the sweep of every non-routed plan: per kernel variant one
// persistent launch over all of its solves, then one finalize per solve.
// Does not synchronise; safe to capture in a CUDA graph.
Status pr_execute_enqueue(std::vector<PrPlan>& plans, PrWorkspace& ws, cudaStream_t stream,
                          int num_sms, bool time_kernels, PrExecReport* rep);

// Pieces of the execution, for callers that schedule item ranges themselves:
// clear a plan's partial slots; one persistent launch over a device table of
// solves (all of one variant) covering n_items items; a plan's final reduction.
Status pr_zero_partials(const PrPlan& P, cudaStream_t stream);
constexpr int kPrVariants = 32;
// Control block of a launch set: one item counter per variant, then the
// error word.
constexpr size_t kPrCtrlErrOffset = 8 * kPrVariants;
constexpr size_t kPrCtrlBytes = kPrCtrlErrOffset + 64;
Status pr_launch(const PrSolve* d_table, int n_solves, long long n_items, int variant,
                 unsigned long long* d_counter, int* d_err, cudaStream_t stream, int num_sms,
                 int max_ctas_per_sm, const PrCtl& ctl = PrCtl{});
Status pr_finalize(const PrPlan& P, cudaStream_t stream);

// After the stream is synchronised: error flag and chunk counts.
Status pr_execute_finish(std::vector<PrPlan>& plans, PrWorkspace& ws, PrExecReport* rep);

}  // namespace xk
