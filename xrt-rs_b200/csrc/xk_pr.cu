// FP32 phase-reduced Kirchhoff path.
//
// Phase decomposition. For a screen tile t (centre P0) and a ray chunk c
// (centre R0, all rays of one energy, wavenumber k) write q = p - R0 for a
// screen point p, rho = r - R0 for a ray r, and u = (P0 - R0)/|P0 - R0|.
// Then exactly
//     |p - r| = |q| - u.rho + Delta,
//     Delta   = (|rho_perp|^2 - 2 v.rho) / (|p - r| + |q| - u.rho),
// with v = q - |q| u (|v| <= tile radius) and rho_perp = rho - (u.rho) u.
// The denominator equals 2(|q| - u.rho) + Delta, and Delta/|q| is far below
// FP32 resolution, so the kernel uses 2(|q| - u.rho).
//   * exp(i k |q|)      per screen point and chunk, FP64 (reference path
//                       length and restored base phase),
//   * exp(-i k u.rho)   per ray and item, FP64 argument reduction folded
//                       into the ray's amplitudes,
//   * exp(i k Delta)    per pair, FP32: |k Delta| <= phase_budget by
//                       construction of the chunk grid.
// This generalises the reference's single-centroid reduction
// (src/gpu/shaders/kirchhoff.wgsl:95-113, src/gpu/kirchhoff.rs:96-104,
// 276-297), whose FP32 residual is unbounded at high Fresnel numbers.
//
// Work decomposition. Screen points are sorted along a Morton curve and cut
// into tiles of 32*kPrPpl points (one warp, kPrPpl points per lane). Rays are
// binned into a grid of cells sized so that the residual phase bound holds
// for every (tile, cell) pair; each occupied cell is a chunk. The sorted ray
// list is cut into `groups` equal ranges; an item is (tile, range), and the
// persistent kernel's warps claim items from an atomic counter. Inside an
// item the range is streamed through shared memory 64 rays at a time by
// cp.async.bulk (TMA bulk copy, mbarrier completion, two buffers), prepared
// in place for the item's direction u, and swept by all 32 lanes. Each lane
// keeps per-point FP32 partial sums folded every stage into two-float
// (TwoSum) accumulators; at a chunk boundary they are multiplied by the FP64
// per-point phasor and added to the item's FP64 slot. A final pass adds the
// `groups` slots of every point in order, so results are deterministic.

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "xk_pr.cuh"

namespace xk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kSumFields = 26;
constexpr uint32_t kMaxWaitIters = 1u << 24;

// ---------------------------------------------------------------------------
// Planner kernels
// ---------------------------------------------------------------------------

enum : int { OP_SUM = 0, OP_MIN = 1, OP_MAX = 2 };
__constant__ int c_sum_ops[kSumFields] = {
    OP_SUM, OP_SUM, OP_SUM,  // ray position sums
    OP_MIN, OP_MIN, OP_MIN, OP_MAX, OP_MAX, OP_MAX,  // ray bbox
    OP_MIN, OP_MAX,                                  // energy range
    OP_MIN, OP_MIN, OP_MIN, OP_MAX, OP_MAX, OP_MAX,  // normal range
    OP_SUM, OP_SUM, OP_SUM,                          // screen position sums
    OP_MIN, OP_MIN, OP_MIN, OP_MAX, OP_MAX, OP_MAX}; // screen bbox

__device__ __forceinline__ double op_combine(int op, double a, double b) {
    return op == OP_SUM ? a + b : (op == OP_MIN ? fmin(a, b) : fmax(a, b));
}

// One partial summary per block over rays and screen points.
__global__ void __launch_bounds__(256) summary_kernel(RaysDev r, int n, PixDev p, int m,
                                                     double* __restrict__ block_out) {
    double f[kSumFields];
    for (int i = 0; i < kSumFields; ++i)
        f[i] = c_sum_ops[i] == OP_SUM ? 0.0 : (c_sum_ops[i] == OP_MIN ? INFINITY : -INFINITY);
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double x = r.x[i], y = r.y[i], z = r.z[i], e = r.energy[i];
        double a = r.nx[i], b = r.ny[i], c = r.nz[i];
        f[0] += x; f[1] += y; f[2] += z;
        f[3] = fmin(f[3], x); f[4] = fmin(f[4], y); f[5] = fmin(f[5], z);
        f[6] = fmax(f[6], x); f[7] = fmax(f[7], y); f[8] = fmax(f[8], z);
        f[9] = fmin(f[9], e); f[10] = fmax(f[10], e);
        f[11] = fmin(f[11], a); f[12] = fmin(f[12], b); f[13] = fmin(f[13], c);
        f[14] = fmax(f[14], a); f[15] = fmax(f[15], b); f[16] = fmax(f[16], c);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        double x = p.x[i], y = p.y[i], z = p.z[i];
        f[17] += x; f[18] += y; f[19] += z;
        f[20] = fmin(f[20], x); f[21] = fmin(f[21], y); f[22] = fmin(f[22], z);
        f[23] = fmax(f[23], x); f[24] = fmax(f[24], y); f[25] = fmax(f[25], z);
    }
    __shared__ double sm[8][kSumFields];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = 0; i < kSumFields; ++i) {
        double v = f[i];
        for (int o = 16; o > 0; o >>= 1) v = op_combine(c_sum_ops[i], v, __shfl_xor_sync(kFull, v, o));
        if (lane == 0) sm[warp][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < kSumFields) {
        int i = threadIdx.x;
        double v = sm[0][i];
        for (int w = 1; w < 8; ++w) v = op_combine(c_sum_ops[i], v, sm[w][i]);
        block_out[blockIdx.x * kSumFields + i] = v;
    }
}

struct Frame {
    double ox, oy, oz;  // origin
    double e1[3], e2[3], u0[3];
    double lo[3], scale[3];  // quantisation: key_a = (coord_a - lo_a) * scale_a
};

__device__ __forceinline__ void to_frame(const Frame& fr, double x, double y, double z,
                                         double out[3]) {
    double dx = x - fr.ox, dy = y - fr.oy, dz = z - fr.oz;
    out[0] = dx * fr.e1[0] + dy * fr.e1[1] + dz * fr.e1[2];
    out[1] = dx * fr.e2[0] + dy * fr.e2[1] + dz * fr.e2[2];
    out[2] = dx * fr.u0[0] + dy * fr.u0[1] + dz * fr.u0[2];
}

__device__ __forceinline__ uint64_t spread21(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

__device__ __forceinline__ uint64_t quant21(double v) {
    double q = floor(v);
    q = fmin(fmax(q, 0.0), 2097151.0);
    return (uint64_t)q;
}

// Morton key of every screen point in the frame.
__global__ void pixel_keys_kernel(PixDev p, int m, Frame fr, uint64_t* __restrict__ keys,
                                  int* __restrict__ idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    double c[3];
    to_frame(fr, p.x[i], p.y[i], p.z[i], c);
    uint64_t k = spread21(quant21((c[0] - fr.lo[0]) * fr.scale[0])) |
                 spread21(quant21((c[1] - fr.lo[1]) * fr.scale[1])) << 1 |
                 spread21(quant21((c[2] - fr.lo[2]) * fr.scale[2])) << 2;
    keys[i] = k;
    idx[i] = i;
}

// One warp per tile: slot table, bounding-box centre, radius.
__global__ void tile_kernel(PixDev p, int m, int n_tiles, const int* __restrict__ sorted_idx,
                            int* __restrict__ tile_perm, double* __restrict__ tile_center,
                            unsigned long long* __restrict__ amax_bits) {
    int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (t >= n_tiles) return;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < kPrPpl; ++i) {
        long long s = (long long)t * kPrTile + lane + 32 * i;
        int id = s < m ? sorted_idx[s] : -1;
        tile_perm[s] = id;
        if (id >= 0) {
            double v[3] = {p.x[id], p.y[id], p.z[id]};
            for (int a = 0; a < 3; ++a) {
                lo[a] = fmin(lo[a], v[a]);
                hi[a] = fmax(hi[a], v[a]);
            }
        }
    }
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fmin(lo[a], __shfl_xor_sync(kFull, lo[a], o));
            hi[a] = fmax(hi[a], __shfl_xor_sync(kFull, hi[a], o));
        }
    double c[3] = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), 0.5 * (lo[2] + hi[2])};
    double rad = 0.0;
    for (int i = 0; i < kPrPpl; ++i) {
        long long s = (long long)t * kPrTile + lane + 32 * i;
        int id = s < m ? sorted_idx[s] : -1;
        if (id >= 0) {
            double dx = p.x[id] - c[0], dy = p.y[id] - c[1], dz = p.z[id] - c[2];
            rad = fmax(rad, sqrt(dx * dx + dy * dy + dz * dz));
        }
    }
    for (int o = 16; o > 0; o >>= 1) rad = fmax(rad, __shfl_xor_sync(kFull, rad, o));
    if (lane == 0) {
        tile_center[3 * t + 0] = c[0];
        tile_center[3 * t + 1] = c[1];
        tile_center[3 * t + 2] = c[2];
        atomicMax(amax_bits, (unsigned long long)__double_as_longlong(rad));
    }
}

struct CellGrid {
    Frame fr;                 // origin, axes, lo[] (cell-grid origin in frame coords)
    double cell[3];           // cell size per axis
    long long n[3];           // cells per axis
};

__device__ __forceinline__ void cell_of(const CellGrid& g, double x, double y, double z,
                                        long long ic[3]) {
    double c[3];
    to_frame(g.fr, x, y, z, c);
    for (int a = 0; a < 3; ++a) {
        double q = g.cell[a] > 0.0 ? floor((c[a] - g.fr.lo[a]) / g.cell[a]) : 0.0;
        long long v = (long long)q;
        v = v < 0 ? 0 : (v >= g.n[a] ? g.n[a] - 1 : v);
        ic[a] = v;
    }
}

__global__ void ray_keys_kernel(RaysDev r, int n, CellGrid g, uint64_t* __restrict__ keys,
                                int* __restrict__ idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long ic[3];
    cell_of(g, r.x[i], r.y[i], r.z[i], ic);
    keys[i] = (uint64_t)((ic[2] * g.n[1] + ic[1]) * g.n[0] + ic[0]);
    idx[i] = i;
}

__global__ void head_flags_kernel(const uint64_t* __restrict__ keys, int n, int* __restrict__ flags) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void chunk_table_kernel(const uint64_t* __restrict__ keys, const int* __restrict__ flags,
                                   const int* __restrict__ run_id, int n, CellGrid g,
                                   int* __restrict__ chunk_begin, double* __restrict__ chunk_center,
                                   int* __restrict__ n_chunks) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) {
        int c = run_id[i] - 1;
        chunk_begin[c] = i;
        uint64_t k = keys[i];
        long long ix = (long long)(k % (uint64_t)g.n[0]);
        long long iy = (long long)((k / (uint64_t)g.n[0]) % (uint64_t)g.n[1]);
        long long iz = (long long)(k / ((uint64_t)g.n[0] * (uint64_t)g.n[1]));
        double f0 = g.fr.lo[0] + (ix + 0.5) * g.cell[0];
        double f1 = g.fr.lo[1] + (iy + 0.5) * g.cell[1];
        double f2 = g.fr.lo[2] + (iz + 0.5) * g.cell[2];
        const Frame& fr = g.fr;
        chunk_center[3 * c + 0] = fr.ox + f0 * fr.e1[0] + f1 * fr.e2[0] + f2 * fr.u0[0];
        chunk_center[3 * c + 1] = fr.oy + f0 * fr.e1[1] + f1 * fr.e2[1] + f2 * fr.u0[1];
        chunk_center[3 * c + 2] = fr.oz + f0 * fr.e1[2] + f1 * fr.e2[2] + f2 * fr.u0[2];
    }
    if (i == n - 1) {
        int nc = run_id[i];
        *n_chunks = nc;
        chunk_begin[nc] = n;
    }
}

__global__ void records_kernel(RaysDev r, int n, const int* __restrict__ sorted_idx,
                               const int* __restrict__ run_id, const double* __restrict__ chunk_center,
                               PrRawRay* __restrict__ recs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = run_id[i] - 1;
    int o = sorted_idx[i];
    PrRawRay rec;
    rec.rx = r.x[o] - chunk_center[3 * c + 0];
    rec.ry = r.y[o] - chunk_center[3 * c + 1];
    rec.rz = r.z[o] - chunk_center[3 * c + 2];
    rec.es_re = (float)r.es_re[o];
    rec.es_im = (float)r.es_im[o];
    rec.ep_re = (float)r.ep_re[o];
    rec.ep_im = (float)r.ep_im[o];
    rec.nx = (float)r.nx[o];
    rec.ny = (float)r.ny[o];
    rec.nz = (float)r.nz[o];
    rec.nl = (float)r.nl[o];
    rec.pad0 = rec.pad1 = 0.f;
    recs[i] = rec;
}

__global__ void finalize_kernel(const double* __restrict__ partial, int groups, int m,
                                FieldDev out) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m) return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int g = 0; g < groups; ++g) {
        const double* b = partial + (size_t)g * 4 * m;
#pragma unroll
        for (int c = 0; c < 4; ++c) s[c] += b[(size_t)c * m + p];
    }
    out.es_re[p] = s[0];
    out.es_im[p] = s[1];
    out.ep_re[p] = s[2];
    out.ep_im[p] = s[3];
}

// ---------------------------------------------------------------------------
// Persistent kernel
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the barrier phase with an iteration limit; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < kMaxWaitIters; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Error-free sum of hi and x into (hi, lo) (Knuth's TwoSum).
__device__ __forceinline__ void two_sum_acc(float& hi, float& lo, float x) {
    float s = hi + x;
    float bb = s - hi;
    float err = (hi - (s - bb)) + (x - bb);
    hi = s;
    lo += err;
}

// Prepared record in shared memory (in place of the 64-byte raw record):
//   a = {rho_x, rho_y, rho_z, R = k |rho_perp|^2}
//   b = {W = -2 u.rho, G = -2 n.rho, nl, 0}
//   e = {es', ep'} with the per-ray phasor exp(-i k u.rho) applied
//   n = {2 nx, 2 ny, 2 nz, 0}

// Per-warp shared state besides the two ray buffers.
template <int P>
struct WarpShared {
    float hi[P * 4][32];  // two-float accumulators, [point*4 + component][lane]
    float lo[P * 4][32];
    double ux, uy, uz;    // item direction for the current chunk
    double r0x, r0y, r0z; // chunk centre
    uint64_t bar[2];      // mbarriers of the two ray buffers
};

template <int P, bool UNIFORM>
struct LaneState {
    float vx[P], vy[P], vz[P], q2[P];
    float nq[P];                // 2 n.q (UNIFORM)
    float qx[P], qy[P], qz[P];  // q (general normals)
    float acc[P][4];
};

template <int P, bool UNIFORM>
__device__ __forceinline__ void setup_points(const PrSolve& sv, int t, int lane,
                                             const WarpShared<P>& ws, LaneState<P, UNIFORM>& ls) {
    const double p0x = sv.tile_center[3 * t], p0y = sv.tile_center[3 * t + 1],
                 p0z = sv.tile_center[3 * t + 2];
    const double ux = ws.ux, uy = ws.uy, uz = ws.uz;
    const double r0x = ws.r0x, r0y = ws.r0y, r0z = ws.r0z;
#pragma unroll
    for (int i = 0; i < P; ++i) {
        int id = sv.tile_perm[(long long)t * kPrTile + lane + 32 * i];
        double x = id >= 0 ? sv.px[id] : p0x;
        double y = id >= 0 ? sv.py[id] : p0y;
        double z = id >= 0 ? sv.pz[id] : p0z;
        double qx = x - r0x, qy = y - r0y, qz = z - r0z;
        double qn = sqrt(qx * qx + qy * qy + qz * qz);
        double vx = qx - qn * ux, vy = qy - qn * uy, vz = qz - qn * uz;
        ls.vx[i] = (float)(-2.0 * sv.k * vx);
        ls.vy[i] = (float)(-2.0 * sv.k * vy);
        ls.vz[i] = (float)(-2.0 * sv.k * vz);
        ls.q2[i] = (float)(2.0 * qn);
        if (UNIFORM) {
            ls.nq[i] = (float)(2.0 * ((double)sv.unx * qx + (double)sv.uny * qy + (double)sv.unz * qz));
        } else {
            // The prepared record carries 2n, so 2 n.q = (2n).q.
            ls.qx[i] = (float)qx;
            ls.qy[i] = (float)qy;
            ls.qz[i] = (float)qz;
        }
    }
}

// Multiplies the lane's two-float sums by (k/2pi) i exp(i k |q|) in FP64 and
// adds them to the item's slots, then clears the sums.
template <int P>
__device__ __forceinline__ void flush_points(const PrSolve& sv, int t, int g, int lane,
                                             WarpShared<P>& ws) {
    const size_t m = (size_t)sv.n_pix;
    double* base = sv.partial + (size_t)g * 4 * m;
    const double r0x = ws.r0x, r0y = ws.r0y, r0z = ws.r0z;
#pragma unroll 1
    for (int i = 0; i < P; ++i) {
        int id = sv.tile_perm[(long long)t * kPrTile + lane + 32 * i];
        if (id >= 0) {
            double qx = sv.px[id] - r0x, qy = sv.py[id] - r0y, qz = sv.pz[id] - r0z;
            double qn = sqrt(qx * qx + qy * qy + qz * qz);
            double turns = sv.kt * qn;
            double f = turns - rint(turns);
            double sp, cp;
            sincospi(2.0 * f, &sp, &cp);
            double phr = -sv.kt * sp, phi = sv.kt * cp;
            double v[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) v[c] = (double)ws.hi[i * 4 + c][lane] + (double)ws.lo[i * 4 + c][lane];
            base[0 * m + id] += v[0] * phr - v[1] * phi;
            base[1 * m + id] += v[0] * phi + v[1] * phr;
            base[2 * m + id] += v[2] * phr - v[3] * phi;
            base[3 * m + id] += v[2] * phi + v[3] * phr;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) ws.hi[i * 4 + c][lane] = ws.lo[i * 4 + c][lane] = 0.f;
    }
}

// Prepares the stage's rays for the item direction (lane j handles rays
// j, j+32).
template <int P>
__device__ __forceinline__ void prep_stage(PrRawRay* buf, int len, int lane, const PrSolve& sv,
                                           const WarpShared<P>& ws) {
    const double ux = ws.ux, uy = ws.uy, uz = ws.uz;
    for (int j = lane; j < len; j += 32) {
        const PrRawRay r = buf[j];
        double ur = ux * r.rx + uy * r.ry + uz * r.rz;
        double tx = r.rx - ur * ux, ty = r.ry - ur * uy, tz = r.rz - ur * uz;
        double perp2 = tx * tx + ty * ty + tz * tz;
        double turns = -sv.kt * ur;
        double f = turns - rint(turns);
        float sn, cs;
        sincospif(2.0f * (float)f, &sn, &cs);
        float rxf = (float)r.rx, ryf = (float)r.ry, rzf = (float)r.rz;
        float4 a = make_float4(rxf, ryf, rzf, (float)(sv.k * perp2));
        float4 b = make_float4((float)(-2.0 * ur), -2.f * (r.nx * rxf + r.ny * ryf + r.nz * rzf),
                               r.nl, 0.f);
        float4 e = make_float4(r.es_re * cs - r.es_im * sn, r.es_re * sn + r.es_im * cs,
                               r.ep_re * cs - r.ep_im * sn, r.ep_re * sn + r.ep_im * cs);
        float4 nn = make_float4(2.f * r.nx, 2.f * r.ny, 2.f * r.nz, 0.f);
        float4* o = reinterpret_cast<float4*>(buf + j);
        o[0] = a;
        o[1] = b;
        o[2] = e;
        o[3] = nn;
    }
}

// The pair sweep: every lane runs the stage's rays against its P points,
// then folds its FP32 partials into the two-float accumulators.
template <int P, bool UNIFORM>
__device__ __forceinline__ void sweep_stage(const PrRawRay* buf, int len, int lane,
                                            LaneState<P, UNIFORM>& ls, WarpShared<P>& ws) {
    const float4* rec = reinterpret_cast<const float4*>(buf);
#pragma unroll
    for (int i = 0; i < P; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) ls.acc[i][c] = 0.f;
#pragma unroll 1
    for (int j = 0; j < len; ++j) {
        const float4 a = rec[4 * j + 0];
        const float4 b = rec[4 * j + 1];
        const float4 e = rec[4 * j + 2];
        float4 nn = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!UNIFORM) nn = rec[4 * j + 3];
#pragma unroll
        for (int i = 0; i < P; ++i) {
            float num = fmaf(ls.vx[i], a.x, a.w);
            num = fmaf(ls.vy[i], a.y, num);
            num = fmaf(ls.vz[i], a.z, num);
            const float rd = rcp_approx(ls.q2[i] + b.x);
            const float th = num * rd;
            float sn, cs;
            __sincosf(th, &sn, &cs);
            float gq;
            if (UNIFORM) {
                gq = ls.nq[i] + b.y;
            } else {
                gq = fmaf(nn.x, ls.qx[i], fmaf(nn.y, ls.qy[i], fmaf(nn.z, ls.qz[i], b.y)));
            }
            const float obl = fmaf(gq, rd, b.z);
            const float amp = obl * rd;
            const float ac = amp * cs, as = amp * sn;
            ls.acc[i][0] = fmaf(e.x, ac, fmaf(-e.y, as, ls.acc[i][0]));
            ls.acc[i][1] = fmaf(e.x, as, fmaf(e.y, ac, ls.acc[i][1]));
            ls.acc[i][2] = fmaf(e.z, ac, fmaf(-e.w, as, ls.acc[i][2]));
            ls.acc[i][3] = fmaf(e.z, as, fmaf(e.w, ac, ls.acc[i][3]));
        }
    }
#pragma unroll
    for (int i = 0; i < P; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float hi = ws.hi[i * 4 + c][lane], lo = ws.lo[i * 4 + c][lane];
            two_sum_acc(hi, lo, ls.acc[i][c]);
            ws.hi[i * 4 + c][lane] = hi;
            ws.lo[i * 4 + c][lane] = lo;
        }
}

struct WarpPipe {
    PrRawRay* buf[2];
    uint64_t* bar[2];
    uint32_t phase;  // bit b: parity of the next completion of buffer b
};

__device__ __forceinline__ void issue_stage(WarpPipe& wp, int b, const PrRawRay* src, int len,
                                            int lane) {
    if (lane == 0) {
        uint32_t bytes = (uint32_t)len * (uint32_t)sizeof(PrRawRay);
        mbar_arrive_expect_tx(wp.bar[b], bytes);
        bulk_g2s(wp.buf[b], src, bytes, wp.bar[b]);
    }
}

__device__ __forceinline__ int chunk_of(const int* __restrict__ begin, int n_chunks, int pos) {
    int lo = 0, hi = n_chunks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (begin[mid] <= pos) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Processes one (tile, ray-range) item; false if a bounded wait ran out.
template <int P, bool UNIFORM>
__device__ bool process_item(const PrSolve& sv, long long local, WarpPipe& wp, WarpShared<P>& ws,
                             int lane) {
    const int t = (int)(local % sv.n_tiles);
    const int g = (int)(local / sv.n_tiles);
    const long long n = sv.n_rays;
    const int r0 = (int)((long long)g * n / sv.groups);
    const int r1 = (int)((long long)(g + 1) * n / sv.groups);
    if (r0 >= r1) return true;
    const int n_chunks = *sv.n_chunks_dev;
    const int* __restrict__ cb = sv.chunk_begin;

#pragma unroll
    for (int i = 0; i < P * 4; ++i) ws.hi[i][lane] = ws.lo[i][lane] = 0.f;

    LaneState<P, UNIFORM> ls;
    int cur_chunk = -1;
    int pos = r0;
    int c = chunk_of(cb, n_chunks, pos);
    int len = min(kPrStage, min(cb[c + 1], r1) - pos);
    int b = 0;
    issue_stage(wp, b, sv.recs + pos, len, lane);
    while (true) {
        // Next stage: same chunk, or the next one at a chunk boundary.
        const int npos = pos + len;
        int nc = c;
        int nlen = 0;
        if (npos < r1) {
            if (npos >= cb[c + 1]) nc = c + 1;
            nlen = min(kPrStage, min(cb[nc + 1], r1) - npos);
            issue_stage(wp, b ^ 1, sv.recs + npos, nlen, lane);
        }
        const bool ok = mbar_wait(wp.bar[b], (wp.phase >> b) & 1u);
        wp.phase ^= (1u << b);
        if (!ok) {
            // Wait (bounded) for the copy in flight on the other buffer.
            if (nlen > 0) {
                mbar_wait(wp.bar[b ^ 1], (wp.phase >> (b ^ 1)) & 1u);
                wp.phase ^= (1u << (b ^ 1));
            }
            return false;
        }
        if (c != cur_chunk) {
            if (cur_chunk >= 0) flush_points<P>(sv, t, g, lane, ws);
            __syncwarp();
            if (lane == 0) {
                const double p0x = sv.tile_center[3 * t], p0y = sv.tile_center[3 * t + 1],
                             p0z = sv.tile_center[3 * t + 2];
                const double r0x = sv.chunk_center[3 * c], r0y = sv.chunk_center[3 * c + 1],
                             r0z = sv.chunk_center[3 * c + 2];
                const double dx = p0x - r0x, dy = p0y - r0y, dz = p0z - r0z;
                const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
                ws.ux = dx * inv;
                ws.uy = dy * inv;
                ws.uz = dz * inv;
                ws.r0x = r0x;
                ws.r0y = r0y;
                ws.r0z = r0z;
            }
            __syncwarp();
            setup_points<P, UNIFORM>(sv, t, lane, ws, ls);
            cur_chunk = c;
        }
        prep_stage<P>(wp.buf[b], len, lane, sv, ws);
        __syncwarp();
        sweep_stage<P, UNIFORM>(wp.buf[b], len, lane, ls, ws);
        // Order this stage's generic-proxy accesses before the next bulk
        // copy into the same buffer.
        fence_proxy_async();
        __syncwarp();
        if (nlen == 0) break;
        pos = npos;
        c = nc;
        len = nlen;
        b ^= 1;
    }
    flush_points<P>(sv, t, g, lane, ws);
    __syncwarp();
    return true;
}

// Every solve in `solves` must have uniform_normal == UNIFORM.
template <int P, bool UNIFORM>
__global__ void __launch_bounds__(kPrWarpsPerCta * 32, 3)
pr_persistent_kernel(const PrSolve* __restrict__ solves, int n_solves, long long n_items,
                     unsigned long long* __restrict__ counter, int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    PrRawRay* bufs = reinterpret_cast<PrRawRay*>(smem) + warp * 2 * kPrStage;
    WarpShared<P>* wsh = reinterpret_cast<WarpShared<P>*>(
                             smem + kPrWarpsPerCta * 2 * kPrStage * sizeof(PrRawRay)) + warp;
    WarpPipe wp;
    wp.buf[0] = bufs;
    wp.buf[1] = bufs + kPrStage;
    wp.bar[0] = &wsh->bar[0];
    wp.bar[1] = &wsh->bar[1];
    wp.phase = 0;
    if (lane == 0) {
        mbar_init(wp.bar[0], 1);
        mbar_init(wp.bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_proxy_async();
    __syncwarp();
    while (true) {
        long long item = 0;
        if (lane == 0) item = (long long)atomicAdd(counter, 1ull);
        item = __shfl_sync(kFull, item, 0);
        if (item >= n_items) break;
        int s = 0;
        while (s + 1 < n_solves && solves[s + 1].item_begin <= item) ++s;
        const PrSolve& sv = solves[s];
        const long long local = item - sv.item_begin;
        const bool ok = process_item<P, UNIFORM>(sv, local, wp, *wsh, lane);
        if (!ok) {
            if (lane == 0) atomicExch(err, 1);
            break;
        }
    }
}

constexpr size_t kPrSmemBytes = (size_t)kPrWarpsPerCta * 2 * kPrStage * sizeof(PrRawRay) +
                                (size_t)kPrWarpsPerCta * sizeof(WarpShared<kPrPpl>);

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Arena {
    char* base;
    size_t off = 0;
    template <class T>
    T* take(size_t count) {
        off = align_up(off, 256);
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

void normalize3(double v[3]) {
    double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (n > 0) {
        v[0] /= n;
        v[1] /= n;
        v[2] /= n;
    }
}

// Range of a world AABB projected on a unit axis through origin o.
void project_box(const double lo[3], const double hi[3], const double o[3], const double ax[3],
                 double* pmin, double* pmax) {
    double mn = INFINITY, mx = -INFINITY;
    for (int c = 0; c < 8; ++c) {
        double p[3] = {(c & 1) ? hi[0] : lo[0], (c & 2) ? hi[1] : lo[1], (c & 4) ? hi[2] : lo[2]};
        double d = (p[0] - o[0]) * ax[0] + (p[1] - o[1]) * ax[1] + (p[2] - o[2]) * ax[2];
        mn = std::min(mn, d);
        mx = std::max(mx, d);
    }
    *pmin = mn;
    *pmax = mx;
}

double box_distance(const double alo[3], const double ahi[3], const double blo[3],
                    const double bhi[3]) {
    double s = 0;
    for (int a = 0; a < 3; ++a) {
        double gap = std::max(0.0, std::max(blo[a] - ahi[a], alo[a] - bhi[a]));
        s += gap * gap;
    }
    return std::sqrt(s);
}

// Upper bound of |k Delta| for chunk radius b, tile radius a, distance d.
double phase_bound(double k, double a, double b, double d) {
    double den = d - 2.0 * b;
    if (den <= 0) return INFINITY;
    return k * (b * b + 2.0 * a * b) / (2.0 * den);
}

}  // namespace

const char* const kRouteReasons[kRouteReasonCount] = {
    "",
    "no rays",
    "rays of different energies",
    "non-positive energy",
    "ray and screen bounding boxes overlap",
    "no cell size meets the phase budget",
    "ray cell grid too fine"};

Status PrWorkspace::ensure_host(size_t bytes) {
    if (bytes <= host_bytes) return Status::Ok();
    if (host) cudaFreeHost(host);
    host = nullptr;
    host_bytes = 0;
    XK_CUDA_TRY(cudaMallocHost(&host, bytes));
    host_bytes = bytes;
    return Status::Ok();
}

void PrWorkspace::release() {
    arena.release();
    cub_tmp.release();
    solves.release();
    ctrl.release();
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    ev[0] = ev[1] = nullptr;
    if (host) cudaFreeHost(host);
    host = nullptr;
    host_bytes = 0;
}

Status pr_solve_enqueue(const RaysDev& rays, size_t n_rays_, const PixDev& pix, size_t n_pix_,
                        const FieldDev& out, PrWorkspace& ws, cudaStream_t stream, int num_sms,
                        PrReport* rep, const PrOptions& opt) {
    PrReport local;
    PrReport& R = rep ? *rep : local;
    R = PrReport();
    if (n_pix_ == 0) return Status::Ok();
    if (n_rays_ == 0) {
        R.routed_f64 = true;
        R.route_reason = 1;  // no rays
        return Status::Ok();
    }
    if (n_rays_ > (size_t)INT32_MAX / 2 || n_pix_ > (size_t)INT32_MAX / 2)
        return Status::Err(XK_ERR_INVALID, "too many rays or screen points for one solve");
    const int n = (int)n_rays_, m = (int)n_pix_;
    const int n_tiles = (m + kPrTile - 1) / kPrTile;

    // Groups: enough items to keep every warp of the persistent grid busy,
    // at least 4 stages of rays per item, partial slots within 4 GiB.
    int groups = opt.groups;
    if (groups <= 0) {
        long long want_items = (long long)num_sms * 12 * 16;
        groups = (int)std::max<long long>(1, (want_items + n_tiles - 1) / n_tiles);
        groups = std::min(groups, std::max(1, n / (4 * kPrStage)));
        long long cap = (4LL << 30) / (32LL * m);
        groups = (int)std::max<long long>(1, std::min<long long>(groups, cap));
        groups = std::min(groups, 256);
    }
    R.groups = groups;

    // --- arena -----------------------------------------------------------
    const int sum_blocks = std::min(512, std::max(1, 2 * num_sms));
    size_t cub_sort_n = 0, cub_sort_m = 0, cub_scan = 0;
    XK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort_n, (uint64_t*)nullptr,
                                                (uint64_t*)nullptr, (int*)nullptr, (int*)nullptr, n));
    XK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort_m, (uint64_t*)nullptr,
                                                (uint64_t*)nullptr, (int*)nullptr, (int*)nullptr, m));
    XK_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, cub_scan, (int*)nullptr, (int*)nullptr, n));
    XK_TRY(ws.cub_tmp.ensure(std::max(cub_sort_n, std::max(cub_sort_m, cub_scan)) + 256));

    size_t need = 0;
    {
        Arena a{nullptr};
        a.take<double>((size_t)sum_blocks * kSumFields);
        a.take<uint64_t>(m); a.take<uint64_t>(m); a.take<int>(m); a.take<int>(m);
        a.take<int>((size_t)n_tiles * kPrTile); a.take<double>(3 * (size_t)n_tiles);
        a.take<unsigned long long>(1);
        a.take<uint64_t>(n); a.take<uint64_t>(n); a.take<int>(n); a.take<int>(n);
        a.take<int>(n); a.take<int>(n);
        a.take<int>((size_t)n + 1); a.take<double>(3 * (size_t)n); a.take<int>(1);
        a.take<PrRawRay>(n);
        a.take<double>((size_t)groups * 4 * m);
        need = a.off + 256;
    }
    XK_TRY(ws.arena.ensure(need));
    Arena a{ws.arena.as<char>()};
    double* d_sum = a.take<double>((size_t)sum_blocks * kSumFields);
    uint64_t* d_pk_in = a.take<uint64_t>(m);
    uint64_t* d_pk_out = a.take<uint64_t>(m);
    int* d_pi_in = a.take<int>(m);
    int* d_pi_out = a.take<int>(m);
    int* d_tile_perm = a.take<int>((size_t)n_tiles * kPrTile);
    double* d_tile_center = a.take<double>(3 * (size_t)n_tiles);
    unsigned long long* d_amax = a.take<unsigned long long>(1);
    uint64_t* d_rk_in = a.take<uint64_t>(n);
    uint64_t* d_rk_out = a.take<uint64_t>(n);
    int* d_ri_in = a.take<int>(n);
    int* d_ri_out = a.take<int>(n);
    int* d_flags = a.take<int>(n);
    int* d_run = a.take<int>(n);
    int* d_chunk_begin = a.take<int>((size_t)n + 1);
    double* d_chunk_center = a.take<double>(3 * (size_t)n);
    int* d_nchunks = a.take<int>(1);
    PrRawRay* d_recs = a.take<PrRawRay>(n);
    double* d_partial = a.take<double>((size_t)groups * 4 * m);

    // Pinned readback area: block summaries | solve descriptor | status words.
    const size_t host_sum_bytes = align_up((size_t)sum_blocks * kSumFields * sizeof(double), 256);
    XK_TRY(ws.ensure_host(host_sum_bytes + align_up(sizeof(PrSolve), 256) + 256));
    double* h_sum = static_cast<double*>(ws.host);
    PrSolve* h_sv = reinterpret_cast<PrSolve*>(static_cast<char*>(ws.host) + host_sum_bytes);
    int* h_misc = reinterpret_cast<int*>(static_cast<char*>(ws.host) + host_sum_bytes +
                                         align_up(sizeof(PrSolve), 256));

    // --- 1. summary -------------------------------------------------------
    summary_kernel<<<sum_blocks, 256, 0, stream>>>(rays, n, pix, m, d_sum);
    XK_CUDA_TRY(cudaGetLastError());
    XK_CUDA_TRY(cudaMemcpyAsync(h_sum, d_sum, (size_t)sum_blocks * kSumFields * sizeof(double),
                                cudaMemcpyDeviceToHost, stream));
    XK_CUDA_TRY(cudaStreamSynchronize(stream));
    R.kernels += 1;
    double f[kSumFields];
    {
        static const int ops[kSumFields] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 1, 2, 1, 1,
                                            1, 2, 2, 2, 0, 0, 0, 1, 1, 1, 2, 2, 2};
        for (int i = 0; i < kSumFields; ++i) {
            double v = h_sum[i];
            for (int bk = 1; bk < sum_blocks; ++bk) {
                double w = h_sum[bk * kSumFields + i];
                v = ops[i] == 0 ? v + w : (ops[i] == 1 ? std::min(v, w) : std::max(v, w));
            }
            f[i] = v;
        }
    }
    if (!(f[9] == f[10])) {
        R.routed_f64 = true;
        R.route_reason = 2;  // rays of different energies
        return Status::Ok();
    }
    const double energy = f[9];
    const double k = (energy / kChbar) * 1e7;
    if (!(k > 0) || !std::isfinite(k)) {
        R.routed_f64 = true;
        R.route_reason = 3;  // non-positive energy
        return Status::Ok();
    }
    const bool uniform_normal = f[11] == f[14] && f[12] == f[15] && f[13] == f[16];
    const double rlo[3] = {f[3], f[4], f[5]}, rhi[3] = {f[6], f[7], f[8]};
    const double plo[3] = {f[20], f[21], f[22]}, phi[3] = {f[23], f[24], f[25]};
    const double d_lo = box_distance(rlo, rhi, plo, phi);
    if (!(d_lo > 0)) {
        R.routed_f64 = true;
        R.route_reason = 4;  // ray and screen bounding boxes overlap
        return Status::Ok();
    }
    const double rc[3] = {f[0] / n, f[1] / n, f[2] / n};
    const double pc[3] = {f[17] / m, f[18] / m, f[19] / m};

    // Frame: u0 from the ray centroid towards the screen centroid.
    Frame fr{};
    double u0[3] = {pc[0] - rc[0], pc[1] - rc[1], pc[2] - rc[2]};
    if (u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2] == 0) u0[2] = 1;
    normalize3(u0);
    double helper[3] = {std::fabs(u0[0]) < 0.9 ? 1.0 : 0.0, std::fabs(u0[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    double dot = helper[0] * u0[0] + helper[1] * u0[1] + helper[2] * u0[2];
    double e1[3] = {helper[0] - dot * u0[0], helper[1] - dot * u0[1], helper[2] - dot * u0[2]};
    normalize3(e1);
    double e2[3] = {u0[1] * e1[2] - u0[2] * e1[1], u0[2] * e1[0] - u0[0] * e1[2],
                    u0[0] * e1[1] - u0[1] * e1[0]};
    for (int i = 0; i < 3; ++i) {
        fr.e1[i] = e1[i];
        fr.e2[i] = e2[i];
        fr.u0[i] = u0[i];
    }

    // --- 2. screen tiles ----------------------------------------------------
    {
        Frame pf = fr;
        pf.ox = pc[0]; pf.oy = pc[1]; pf.oz = pc[2];
        const double* axes[3] = {e1, e2, u0};
        for (int ax = 0; ax < 3; ++ax) {
            double mn, mx;
            project_box(plo, phi, pc, axes[ax], &mn, &mx);
            pf.lo[ax] = mn;
            pf.scale[ax] = (mx > mn) ? 2097151.0 / (mx - mn) : 0.0;
        }
        pixel_keys_kernel<<<(m + 255) / 256, 256, 0, stream>>>(pix, m, pf, d_pk_in, d_pi_in);
        XK_CUDA_TRY(cudaGetLastError());
        size_t tmp = ws.cub_tmp.bytes;
        XK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp.ptr, tmp, d_pk_in, d_pk_out, d_pi_in,
                                                    d_pi_out, m, 0, 63, stream));
        XK_CUDA_TRY(cudaMemsetAsync(d_amax, 0, sizeof(unsigned long long), stream));
        int warps_blocks = (n_tiles * 32 + 255) / 256;
        tile_kernel<<<warps_blocks, 256, 0, stream>>>(pix, m, n_tiles, d_pi_out, d_tile_perm,
                                                       d_tile_center, d_amax);
        XK_CUDA_TRY(cudaGetLastError());
        XK_CUDA_TRY(cudaMemcpyAsync(h_sum, d_amax, sizeof(double), cudaMemcpyDeviceToHost, stream));
        XK_CUDA_TRY(cudaStreamSynchronize(stream));
        R.kernels += 2;
    }
    const double a_max = h_sum[0] * 1.001;

    // --- 3. ray cells -----------------------------------------------------
    CellGrid cg{};
    cg.fr = fr;
    cg.fr.ox = rc[0]; cg.fr.oy = rc[1]; cg.fr.oz = rc[2];
    double ext[3];
    {
        const double* axes[3] = {e1, e2, u0};
        for (int ax = 0; ax < 3; ++ax) {
            double mn, mx;
            project_box(rlo, rhi, rc, axes[ax], &mn, &mx);
            cg.fr.lo[ax] = mn;
            ext[ax] = mx - mn;
        }
    }
    auto cell_radius = [&](double h, double cell[3]) {
        double s = 0;
        for (int ax = 0; ax < 3; ++ax) {
            cell[ax] = ext[ax] <= h ? ext[ax] : h;
            s += 0.25 * cell[ax] * cell[ax];
        }
        return std::sqrt(s);
    };
    double cell[3];
    double h_hi = 2.0 * std::max(ext[0], std::max(ext[1], ext[2])) + 1e-300;
    double h_lo = 0.0;
    if (phase_bound(k, a_max, cell_radius(h_hi, cell), d_lo) <= opt.phase_budget) {
        h_lo = h_hi;
    } else {
        for (int it = 0; it < 200; ++it) {
            double h = 0.5 * (h_lo + h_hi);
            if (phase_bound(k, a_max, cell_radius(h, cell), d_lo) <= opt.phase_budget) h_lo = h;
            else h_hi = h;
        }
    }
    const double h = h_lo;
    const double b_max = cell_radius(h, cell);
    if (!(h > 0)) {
        R.routed_f64 = true;
        R.route_reason = 5;  // no cell size meets the phase budget
        return Status::Ok();
    }
    for (int ax = 0; ax < 3; ++ax) {
        cg.cell[ax] = cell[ax];
        double cnt = cell[ax] > 0 ? std::floor(ext[ax] / cell[ax]) + 1.0 : 1.0;
        if (cnt > 2097151.0) {
            R.routed_f64 = true;
            R.route_reason = 6;  // ray cell grid too fine
            return Status::Ok();
        }
        cg.n[ax] = (long long)cnt;
    }
    R.phase_bound = phase_bound(k, a_max, b_max, d_lo);

    ray_keys_kernel<<<(n + 255) / 256, 256, 0, stream>>>(rays, n, cg, d_rk_in, d_ri_in);
    XK_CUDA_TRY(cudaGetLastError());
    {
        size_t tmp = ws.cub_tmp.bytes;
        XK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp.ptr, tmp, d_rk_in, d_rk_out, d_ri_in,
                                                    d_ri_out, n, 0, 63, stream));
    }
    head_flags_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_rk_out, n, d_flags);
    XK_CUDA_TRY(cudaGetLastError());
    {
        size_t tmp = ws.cub_tmp.bytes;
        XK_CUDA_TRY(cub::DeviceScan::InclusiveSum(ws.cub_tmp.ptr, tmp, d_flags, d_run, n, stream));
    }
    chunk_table_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_rk_out, d_flags, d_run, n, cg,
                                                             d_chunk_begin, d_chunk_center, d_nchunks);
    XK_CUDA_TRY(cudaGetLastError());
    records_kernel<<<(n + 255) / 256, 256, 0, stream>>>(rays, n, d_ri_out, d_run, d_chunk_center,
                                                         d_recs);
    XK_CUDA_TRY(cudaGetLastError());
    R.kernels += 5;

    // --- 4. persistent sweep ------------------------------------------------
    PrSolve sv{};
    sv.recs = d_recs;
    sv.chunk_begin = d_chunk_begin;
    sv.chunk_center = d_chunk_center;
    sv.n_chunks_dev = d_nchunks;
    sv.tile_perm = d_tile_perm;
    sv.tile_center = d_tile_center;
    sv.px = pix.x;
    sv.py = pix.y;
    sv.pz = pix.z;
    sv.partial = d_partial;
    sv.item_begin = 0;
    sv.n_items = (long long)n_tiles * groups;
    sv.n_rays = n;
    sv.n_pix = m;
    sv.n_tiles = n_tiles;
    sv.groups = groups;
    sv.k = k;
    sv.kt = k / (2.0 * kPi);
    sv.uniform_normal = uniform_normal ? 1 : 0;
    {
        // The common normal, read back from the summary (min == max).
        sv.unx = (float)f[11];
        sv.uny = (float)f[12];
        sv.unz = (float)f[13];
    }
    XK_TRY(ws.solves.ensure(sizeof(PrSolve)));
    XK_TRY(ws.ctrl.ensure(64));
    *h_sv = sv;
    XK_CUDA_TRY(cudaMemcpyAsync(ws.solves.ptr, h_sv, sizeof(PrSolve), cudaMemcpyHostToDevice, stream));
    XK_CUDA_TRY(cudaMemsetAsync(ws.ctrl.ptr, 0, 64, stream));
    XK_CUDA_TRY(cudaMemsetAsync(d_partial, 0, (size_t)groups * 4 * m * sizeof(double), stream));

    auto kern = uniform_normal ? pr_persistent_kernel<kPrPpl, true>
                               : pr_persistent_kernel<kPrPpl, false>;
    XK_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kPrSmemBytes));
    int per_sm = 0;
    XK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPrWarpsPerCta * 32,
                                                              kPrSmemBytes));
    per_sm = std::max(per_sm, 1);
    long long grid = (long long)num_sms * per_sm;
    long long max_ctas = (sv.n_items + kPrWarpsPerCta - 1) / kPrWarpsPerCta;
    grid = std::max<long long>(1, std::min(grid, max_ctas));
    unsigned long long* d_counter = reinterpret_cast<unsigned long long*>(ws.ctrl.ptr);
    int* d_err = reinterpret_cast<int*>(static_cast<char*>(ws.ctrl.ptr) + 8);
    if (!ws.ev[0]) XK_CUDA_TRY(cudaEventCreate(&ws.ev[0]));
    if (!ws.ev[1]) XK_CUDA_TRY(cudaEventCreate(&ws.ev[1]));
    XK_CUDA_TRY(cudaEventRecord(ws.ev[0], stream));
    kern<<<(unsigned)grid, kPrWarpsPerCta * 32, kPrSmemBytes, stream>>>(
        reinterpret_cast<const PrSolve*>(ws.solves.ptr), 1, sv.n_items, d_counter, d_err);
    XK_CUDA_TRY(cudaGetLastError());
    XK_CUDA_TRY(cudaEventRecord(ws.ev[1], stream));
    finalize_kernel<<<(m + 255) / 256, 256, 0, stream>>>(d_partial, groups, m, out);
    XK_CUDA_TRY(cudaGetLastError());
    R.kernels += 2;

    XK_CUDA_TRY(cudaMemcpyAsync(h_misc, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    XK_CUDA_TRY(cudaMemcpyAsync(h_misc + 1, d_nchunks, sizeof(int), cudaMemcpyDeviceToHost, stream));
    XK_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h_misc[0] != 0)
        return Status::Err(XK_ERR_TIMEOUT, "persistent kernel: bounded wait for a ray stage ran out");
    XK_CUDA_TRY(cudaEventElapsedTime(&R.main_kernel_ms, ws.ev[0], ws.ev[1]));
    R.n_tiles = n_tiles;
    R.n_chunks = h_misc[1];
    R.n_items = sv.n_items;
    return Status::Ok();
}

}  // namespace xk
