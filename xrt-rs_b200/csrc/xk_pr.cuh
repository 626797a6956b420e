// FP32 phase-reduced Kirchhoff path: planner + persistent kernel.
#pragma once

#include "xk_internal.cuh"

namespace xk {

// Geometry of the work decomposition.
constexpr int kPrWarpsPerCta = 4;
constexpr int kPrStage = 64;          // rays per shared-memory stage
constexpr int kPrPpl = 8;             // screen points per lane
constexpr int kPrTile = 32 * kPrPpl;  // screen points per tile (one warp)

// Planner knobs.
struct PrOptions {
    double phase_budget = 256.0;  // bound on |FP32 residual phase| [rad]
    double min_rays_per_chunk = 2.0;
    int groups = 0;  // ray groups per tile; 0 = automatic
};

struct PrReport {
    int kernels = 0;
    bool routed_f64 = false;
    int route_reason = 0;  // index into kRouteReasons
    int n_tiles = 0;
    int n_chunks = 0;
    long long n_items = 0;
    double phase_bound = 0.0;
    int groups = 0;
    float main_kernel_ms = 0.f;
};

// Reasons a solve is routed to the FP64 path (xk_route_reason).
constexpr int kRouteReasonCount = 7;
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

// Device-side description of one planned solve.
struct PrSolve {
    const PrRawRay* recs;         // [n_rays] in chunk order
    const int* chunk_begin;       // [n_chunks + 1]
    const double* chunk_center;   // [3 * n_chunks]
    const int* n_chunks_dev;      // scalar
    const int* tile_perm;         // [n_tiles * kPrTile], -1 = padding slot
    const double* tile_center;    // [3 * n_tiles]
    const double *px, *py, *pz;   // screen points (original order)
    double* partial;              // [groups][4][n_pix]
    long long item_begin;         // first global item of this solve
    long long n_items;            // n_tiles * groups
    int n_rays, n_pix, n_tiles, groups;
    double k;                     // wavenumber [1/mm]
    double kt;                    // k / (2 pi)  (turns per mm)
    int uniform_normal;
    float unx, uny, unz;          // the common normal when uniform_normal
};

struct PrWorkspace {
    DevBuf arena;
    DevBuf cub_tmp;
    DevBuf solves;  // PrSolve array for the persistent launch
    DevBuf ctrl;    // counter + error flag
    cudaEvent_t ev[2] = {nullptr, nullptr};  // bracket the pair kernel
    void* host = nullptr;  // pinned readback area
    size_t host_bytes = 0;
    Status ensure_host(size_t bytes);
    void release();
};

Status pr_solve_enqueue(const RaysDev& rays, size_t n_rays, const PixDev& pix, size_t n_pix,
                        const FieldDev& out, PrWorkspace& ws, cudaStream_t stream, int num_sms,
                        PrReport* rep, const PrOptions& opt = PrOptions());

}  // namespace xk
