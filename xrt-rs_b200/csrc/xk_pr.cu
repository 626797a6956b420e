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
//   * exp(i k |q|)      per screen point and chunk: reference path length and
//                       its turn count in FP64, sin/cos of the reduced turn,
//   * exp(-i k u.rho)   per ray and item, FP64 argument reduction folded
//                       into the ray's amplitudes,
//   * exp(i k Delta)    per pair, FP32: |k Delta| <= the residual-phase
//                       budget by construction of the chunk grid (the budget
//                       follows from the requested tolerance).
// This generalises the reference's single-centroid reduction
// (src/gpu/shaders/kirchhoff.wgsl:95-113, src/gpu/kirchhoff.rs:96-104,
// 276-297), whose FP32 residual is unbounded at high Fresnel numbers.
//
// Work decomposition. Screen points are sorted along a Hilbert curve and cut
// into tiles of 32*kPrPpl points (one warp, kPrPpl points per lane). Rays are
// binned into a grid of cells sized so that the residual phase bound holds
// for every (tile, cell) pair; each occupied cell is a chunk. The sorted ray
// list is cut into `groups` equal ranges; an item is (tile, range), and the
// persistent kernel's warps claim items from an atomic counter. Inside an
// item the range is streamed through shared memory kPrStage rays at a time by
// cp.async.bulk (TMA bulk copy, mbarrier completion, two buffers), prepared
// in place for the item's direction u, and swept by all 32 lanes. Each lane
// keeps per-point FP32 partial sums folded every stage into two-float
// (TwoSum) accumulators; at a chunk boundary they are multiplied by the
// per-point phasor and added, in FP64, to the item's slot. A final pass adds
// the `groups` slots of every point in order, so results are deterministic.
//
// Two sweeps: the SFU sweep (rcp.approx for 1/(2|q| - 2u.rho)) and the packed
// sweep, which processes two screen points per instruction with the sm_100
// f32x2 FMA and replaces the reciprocal by the series
// r0 (1 + e + e^2), r0 = 1/(2|q|), e = 2u.rho r0, when the planner can bound
// |e| (the neglected e^3 term then stays below 1e-8 relative).

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "xk_pr.cuh"
#include "xk_sm100.cuh"

namespace xk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kSumFields = 33;
// Stages of FP32 partial sums per fold into the two-float accumulators.
constexpr int kFoldStages = 1;
// |e| bound under which the packed sweep's series reciprocal is used.
constexpr double kSeriesRcpBound = 2e-3;
// Fold the base phase when the estimated chunks per ray group reach this.
constexpr double kFoldChunksPerGroup = 4.0;
// ... and chunks average fewer rays than this: a chunk switch (the points'
// double-double base phase and the flush of the chunk sums) costs about as
// much as sweeping 30 rays, the folded sweep about 8 % more per ray.
constexpr double kFoldRaysPerChunk = 512.0;
// Largest |es_j ep_0 - ep_j es_0| / (|es_j| |ep_0| + |ep_j| |es_0|) over the
// rays under which every ray counts as having ray 0's polarization (2^-24:
// the per-ray deviation is then below the FP32 rounding of the amplitudes
// that the kernel applies anyway).
constexpr double kOnePolTol = 5.9604644775390625e-8;
// Amplitude components the phase-reduced kernels carry in FP32: their partial
// sums over a chunk (up to 2^20 rays, |U| up to ~1/path) must stay inside
// FP32's range, and products with |U| must stay normal.
constexpr double kF32AmpMax = 1e30, kF32AmpMin = 1e-30;

// ---------------------------------------------------------------------------
// Planner kernels
// ---------------------------------------------------------------------------

enum : int { OP_SUM = 0, OP_MIN = 1, OP_MAX = 2 };
__constant__ int c_sum_ops[kSumFields] = {
    OP_SUM, OP_SUM, OP_SUM,                          // ray position sums
    OP_MIN, OP_MIN, OP_MIN, OP_MAX, OP_MAX, OP_MAX,  // ray bbox
    OP_MIN, OP_MAX,                                  // energy range
    OP_MIN, OP_MIN, OP_MIN, OP_MAX, OP_MAX, OP_MAX,  // normal range
    OP_SUM, OP_SUM, OP_SUM,                          // screen position sums
    OP_MIN, OP_MIN, OP_MIN, OP_MAX, OP_MAX, OP_MAX,  // screen bbox
    OP_SUM,                                          // non-finite probe
    OP_MAX,                                          // polarization deviation
    OP_SUM, OP_SUM, OP_SUM, OP_SUM,                  // ray 0's es, ep
    OP_MAX};                                         // largest amplitude component
const int h_sum_ops[kSumFields] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 1, 2, 1, 1, 1, 2, 2, 2,
                                   0, 0, 0, 1, 1, 1, 2, 2, 2, 0, 2, 0, 0, 0, 0, 2};

__device__ __forceinline__ double op_combine(int op, double a, double b) {
    return op == OP_SUM ? a + b : (op == OP_MIN ? fmin(a, b) : fmax(a, b));
}

// One partial summary per block over rays and screen points. The last field
// sums every input value times zero: 0 when all are finite, NaN otherwise
// (fmin / fmax skip NaN, so the boxes alone would not show it). Fields 27-31
// test whether all rays share ray 0's polarization: the largest relative
// |es_j ep_0 - ep_j es_0|, and ray 0's (es, ep); field 32 is the largest
// amplitude component.
__global__ void __launch_bounds__(256) summary_kernel(RaysDev r, int n, PixDev p, int m,
                                                     double* __restrict__ block_out) {
    double f[kSumFields];
    for (int i = 0; i < kSumFields; ++i)
        f[i] = c_sum_ops[i] == OP_SUM ? 0.0 : (c_sum_ops[i] == OP_MIN ? INFINITY : -INFINITY);
    const int stride = gridDim.x * blockDim.x;
    const double a0r = r.es_re[0], a0i = r.es_im[0], b0r = r.ep_re[0], b0i = r.ep_im[0];
    const double a0n = sqrt(a0r * a0r + a0i * a0i), b0n = sqrt(b0r * b0r + b0i * b0i);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double x = r.x[i], y = r.y[i], z = r.z[i], e = r.energy[i];
        double a = r.nx[i], b = r.ny[i], c = r.nz[i];
        f[0] += x; f[1] += y; f[2] += z;
        f[3] = fmin(f[3], x); f[4] = fmin(f[4], y); f[5] = fmin(f[5], z);
        f[6] = fmax(f[6], x); f[7] = fmax(f[7], y); f[8] = fmax(f[8], z);
        f[9] = fmin(f[9], e); f[10] = fmax(f[10], e);
        f[11] = fmin(f[11], a); f[12] = fmin(f[12], b); f[13] = fmin(f[13], c);
        f[14] = fmax(f[14], a); f[15] = fmax(f[15], b); f[16] = fmax(f[16], c);
        const double ar = r.es_re[i], ai = r.es_im[i], br = r.ep_re[i], bi = r.ep_im[i];
        f[26] += (x + y + z + e + a + b + c + r.nl[i] + ar + ai + br + bi) * 0.0;
        const double dr = (ar * b0r - ai * b0i) - (br * a0r - bi * a0i);
        const double di = (ar * b0i + ai * b0r) - (br * a0i + bi * a0r);
        const double nrm = sqrt(ar * ar + ai * ai) * b0n + sqrt(br * br + bi * bi) * a0n;
        const double dn = sqrt(dr * dr + di * di);
        f[27] = fmax(f[27], nrm > 0.0 ? dn / nrm : (dn > 0.0 ? INFINITY : 0.0));
        f[32] = fmax(f[32], fmax(fmax(fabs(ar), fabs(ai)), fmax(fabs(br), fabs(bi))));
        if (i == 0) {
            f[28] += ar;
            f[29] += ai;
            f[30] += br;
            f[31] += bi;
        }
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        double x = p.x[i], y = p.y[i], z = p.z[i];
        f[17] += x; f[18] += y; f[19] += z;
        f[20] = fmin(f[20], x); f[21] = fmin(f[21], y); f[22] = fmin(f[22], z);
        f[23] = fmax(f[23], x); f[24] = fmax(f[24], y); f[25] = fmax(f[25], z);
        f[26] += (x + y + z) * 0.0;
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
    double lo[3], scale[3];  // quantisation: q_a = (coord_a - lo_a) * scale_a
};

__device__ __forceinline__ void to_frame(const Frame& fr, double x, double y, double z,
                                         double out[3]) {
    double dx = x - fr.ox, dy = y - fr.oy, dz = z - fr.oz;
    out[0] = dx * fr.e1[0] + dy * fr.e1[1] + dz * fr.e1[2];
    out[1] = dx * fr.e2[0] + dy * fr.e2[1] + dz * fr.e2[2];
    out[2] = dx * fr.u0[0] + dy * fr.u0[1] + dz * fr.u0[2];
}

__device__ __forceinline__ uint32_t quant(double v, double maxv) {
    double q = floor(v);
    q = fmin(fmax(q, 0.0), maxv);
    return (uint32_t)q;
}

// Distance of (x, y) along the Hilbert curve of order 16 (the classic
// iterative xy -> d mapping: quadrant digit per level, then rotate/flip).
__device__ __forceinline__ uint32_t hilbert16(uint32_t x, uint32_t y) {
    uint32_t d = 0;
    for (uint32_t s = 1u << 15; s > 0; s >>= 1) {
        uint32_t rx = (x & s) ? 1u : 0u;
        uint32_t ry = (y & s) ? 1u : 0u;
        d += s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = 0xffffu - x;
                y = 0xffffu - y;
            }
            uint32_t t = x;
            x = y;
            y = t;
        }
    }
    return d;
}

// Hilbert key of every screen point over its two transverse frame axes, the
// longitudinal coordinate as tie-break.
__global__ void pixel_keys_kernel(PixDev p, int m, Frame fr, uint64_t* __restrict__ keys,
                                  int* __restrict__ idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    double c[3];
    to_frame(fr, p.x[i], p.y[i], p.z[i], c);
    uint32_t hx = quant((c[0] - fr.lo[0]) * fr.scale[0], 65535.0);
    uint32_t hy = quant((c[1] - fr.lo[1]) * fr.scale[1], 65535.0);
    uint32_t hz = quant((c[2] - fr.lo[2]) * fr.scale[2], 2097151.0);
    keys[i] = ((uint64_t)hilbert16(hx, hy) << 21) | hz;
    idx[i] = i;
}

// One warp per tile: slot table, slot-ordered coordinates, bounding-box
// centre, radius.
__global__ void tile_kernel(PixDev p, int m, int n_tiles, const int* __restrict__ sorted_idx,
                            int* __restrict__ tile_perm, double* __restrict__ tpx,
                            double* __restrict__ tpy, double* __restrict__ tpz,
                            double* __restrict__ tile_center,
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
        double x = c[0], y = c[1], z = c[2];
        if (id >= 0) {
            x = p.x[id];
            y = p.y[id];
            z = p.z[id];
            double dx = x - c[0], dy = y - c[1], dz = z - c[2];
            rad = fmax(rad, sqrt(dx * dx + dy * dy + dz * dz));
        }
        tpx[s] = x;
        tpy[s] = y;
        tpz[s] = z;
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
    Frame fr;        // origin, axes, lo[] (cell-grid origin in frame coords)
    double cell[3];  // cell size per axis
    long long n[3];  // cells per axis
    double quantum, inv_quantum;  // chunk centres are multiples of quantum (a power of two)
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
        // Snapped to multiples of g.quantum (a power of two no smaller than the
        // ulp of any coordinate in play), so that q = p - R0 is exact: at
        // |p| ~ 2e4 mm one rounding of q is 1.8e-12 mm, 2.8e-4 rad at 30 keV.
        const double cx = fr.ox + f0 * fr.e1[0] + f1 * fr.e2[0] + f2 * fr.u0[0];
        const double cy = fr.oy + f0 * fr.e1[1] + f1 * fr.e2[1] + f2 * fr.u0[1];
        const double cz = fr.oz + f0 * fr.e1[2] + f1 * fr.e2[2] + f2 * fr.u0[2];
        chunk_center[3 * c + 0] = rint(cx * g.inv_quantum) * g.quantum;
        chunk_center[3 * c + 1] = rint(cy * g.inv_quantum) * g.quantum;
        chunk_center[3 * c + 2] = rint(cz * g.inv_quantum) * g.quantum;
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

// Orders the ray groups of a solve by decreasing estimated cost, so that the
// persistent kernel hands out the most expensive (tile, group) items first and
// the launch does not end on a few long ones. A group's cost is its ray count
// plus kGroupChunkCost rays for every chunk it spans (each chunk boundary
// costs a per-point set-up and flush, about the sweep of that many rays).
// One block, bitonic sort of (cost, group) keys in shared memory; ties keep
// group order, so the schedule is deterministic. groups <= kMaxGroups.
constexpr int kMaxGroups = 4096;
constexpr int kGroupChunkCost = 24;

__global__ void __launch_bounds__(1024) group_order_kernel(const int* __restrict__ chunk_begin,
                                                           const int* __restrict__ n_chunks_dev,
                                                           int n, int groups,
                                                           int* __restrict__ order) {
    __shared__ unsigned long long key[kMaxGroups];
    const int n_chunks = *n_chunks_dev;
    int len = 1;
    while (len < groups) len <<= 1;
    auto chunk_at = [&](int pos) {
        int lo = 0, hi = n_chunks - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (chunk_begin[mid] <= pos) lo = mid;
            else hi = mid - 1;
        }
        return lo;
    };
    for (int g = threadIdx.x; g < len; g += blockDim.x) {
        unsigned long long k = ~0ull;
        if (g < groups) {
            const long long r0 = (long long)g * n / groups, r1 = (long long)(g + 1) * n / groups;
            unsigned int cost = 0;
            if (r1 > r0) {
                const int c = chunk_at((int)(r1 - 1)) - chunk_at((int)r0) + 1;
                const long long w = (r1 - r0) + (long long)kGroupChunkCost * c;
                cost = (unsigned int)(w < 0x7fffffffLL ? w : 0x7fffffffLL);
            }
            // Ascending keys = descending cost, then ascending group.
            k = ((unsigned long long)(0xffffffffu - cost) << 32) | (unsigned int)g;
        }
        key[g] = k;
    }
    __syncthreads();
    for (int size = 2; size <= len; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < len; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const unsigned long long a = key[i], b = key[j];
                    if ((a > b) == up) {
                        key[i] = b;
                        key[j] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < groups; i += blockDim.x) order[i] = (int)(key[i] & 0xffffffffu);
}

// Adds the groups' slots of every tile slot in order and scatters the sum to
// the screen point's original index.
// One-polarization solves hold A in components 0 and 1; the field is
// (pes * A, pep * A).
__global__ void finalize_kernel(const double* __restrict__ partial, const int* __restrict__ tile_perm,
                                int groups, int slots, FieldDev out, int one_pol, double2 pes,
                                double2 pep) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slots) return;
    int id = tile_perm[s];
    if (id < 0) return;
    if (one_pol) {
        double ar = 0.0, ai = 0.0;
        for (int g = 0; g < groups; ++g) {
            const double* b = partial + (size_t)g * 4 * slots;
            ar += b[s];
            ai += b[(size_t)slots + s];
        }
        out.es_re[id] = pes.x * ar - pes.y * ai;
        out.es_im[id] = pes.x * ai + pes.y * ar;
        out.ep_re[id] = pep.x * ar - pep.y * ai;
        out.ep_im[id] = pep.x * ai + pep.y * ar;
        return;
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int g = 0; g < groups; ++g) {
        const double* b = partial + (size_t)g * 4 * slots;
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[c] += b[(size_t)c * slots + s];
    }
    out.es_re[id] = acc[0];
    out.es_im[id] = acc[1];
    out.ep_re[id] = acc[2];
    out.ep_im[id] = acc[3];
}

// ---------------------------------------------------------------------------
// Persistent kernel
// ---------------------------------------------------------------------------

using namespace sm100;  // mbarriers with bounded waits, bulk copies (xk_sm100.cuh)

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

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// Prepared record in shared memory (in place of the 64-byte raw record):
//   a = {rho_x, rho_y, rho_z, R = k |rho_perp|^2}
//   b = {W = -2 u.rho, G = -2 n.rho, nl, -W}
//   e = {es', ep'} with the per-ray phasor exp(-i k u.rho) applied
//   n = {2 nx, 2 ny, 2 nz, 0}
//
// Per-warp shared state besides the two ray buffers. NC components per point:
// 4 (Es, Ep) or 2 (the one-polarization kernels' single column), which is
// what lets those kernels fit four CTAs per SM.
template <int NC>
struct WarpSharedT {
    static constexpr int kNC = NC;
    float hi[kPrPpl * NC][32];  // two-float accumulators, [point*NC + component][lane]
    float lo[kPrPpl * NC][32];
    float2 ph[kPrPpl][32];      // (k/2pi) i exp(i k |q|) of the current chunk (unfolded variants)
    double ux, uy, uz;          // item direction for the current chunk
    double r0x, r0y, r0z;       // chunk centre
    uint64_t bar[2];            // mbarriers of the two ray buffers
};

// Per-lane state of the SFU sweep.
template <bool UNIFORM>
struct ScalarState {
    float vx[kPrPpl], vy[kPrPpl], vz[kPrPpl], q2[kPrPpl];  // q2 = 2|q|
    float nq[kPrPpl];                                        // 2 n.q (UNIFORM)
    float qx[kPrPpl], qy[kPrPpl], qz[kPrPpl];                // q (general normals)
    float phi[kPrPpl];                                       // base phase k|q| mod 2 pi
    float acc[kPrPpl][4];
};

// Per-lane state of the packed sweep: point pairs (2i, 2i+1).
template <bool UNIFORM>
struct PackedState {
    float2 vx[kPrPpl / 2], vy[kPrPpl / 2], vz[kPrPpl / 2], q2[kPrPpl / 2];  // q2 = 1/(2|q|)
    float2 nq[kPrPpl / 2];
    float2 qx[kPrPpl / 2], qy[kPrPpl / 2], qz[kPrPpl / 2];
    float2 phi[kPrPpl / 2];  // base phase k|q| mod 2 pi
    float2 acc[kPrPpl / 2][4];
};

// Fractional part of (kt_hi + kt_lo) * |q| in turns, |q| = sqrt(qx^2+qy^2+qz^2),
// evaluated in double-double arithmetic (error-free products by FMA, TwoSum,
// one Newton correction of the square root).
__device__ __forceinline__ double dd_turns(double kt_hi, double kt_lo, double qx, double qy,
                                           double qz, double* qn, double* inv2q) {
    const double p0 = qx * qx, p1 = qy * qy, p2 = qz * qz;
    const double e0 = fma(qx, qx, -p0), e1 = fma(qy, qy, -p1), e2 = fma(qz, qz, -p2);
    double s1 = p0 + p1;
    double b1 = s1 - p0;
    double t1 = (p0 - (s1 - b1)) + (p1 - b1);
    double s2 = s1 + p2;
    double b2 = s2 - s1;
    double t2 = (s1 - (s2 - b2)) + (p2 - b2);
    double lo = t1 + t2 + e0 + e1 + e2;
    double hi = s2 + lo;
    lo -= hi - s2;
    const double r = sqrt(hi);
    *qn = r;
    // 1/(2r): f32 reciprocal seed and one FP64 Newton step (~1e-14 relative);
    // it scales the square root's low-order correction and is the sweep's
    // 1/(2|q|).
    const double d2 = 2.0 * r;
    const double y0 = (double)__frcp_rn((float)d2);
    const double y = fma(y0, fma(-d2, y0, 1.0), y0);
    *inv2q = y;
    const double rl = (fma(-r, r, hi) + lo) * y;
    const double ph = kt_hi * r;
    const double pe = fma(kt_hi, r, -ph) + (kt_hi * rl + kt_lo * r);
    return (ph - rint(ph)) + pe;
}

// Per chunk: FP64 geometry of the lane's points, written into the sweep
// state, and the per-point base phase k|q|: folded into the sweep state
// (FOLD) or as the chunk phasor (k/2pi) i exp(i k|q|) into shared memory.
template <bool UNIFORM, bool FAST, bool FOLD, class State, class WS>
__device__ __forceinline__ void setup_points(const PrSolve& sv, int t, int lane, WS& ws,
                                             State& st) {
    const double ux = ws.ux, uy = ws.uy, uz = ws.uz;
    const double r0x = ws.r0x, r0y = ws.r0y, r0z = ws.r0z;
    const double k = sv.k;
    float* vxp = reinterpret_cast<float*>(st.vx);
    float* vyp = reinterpret_cast<float*>(st.vy);
    float* vzp = reinterpret_cast<float*>(st.vz);
    float* q2p = reinterpret_cast<float*>(st.q2);
    float* nqp = reinterpret_cast<float*>(st.nq);
    float* qxp = reinterpret_cast<float*>(st.qx);
    float* qyp = reinterpret_cast<float*>(st.qy);
    float* qzp = reinterpret_cast<float*>(st.qz);
#pragma unroll
    for (int i = 0; i < kPrPpl; ++i) {
        const long long s = (long long)t * kPrTile + lane + 32 * i;
        double qx = sv.tpx[s] - r0x, qy = sv.tpy[s] - r0y, qz = sv.tpz[s] - r0z;
        // Base phase k|q| in turns, carried in double-double (k|q| reaches
        // 1e12 rad at 30 keV and 20 m, where one FP64 rounding is 1e-4 rad);
        // the same square root gives |q|.
        double qn, inv2q;
        const float fr = (float)dd_turns(sv.kt, sv.kt_lo, qx, qy, qz, &qn, &inv2q);
        double vx = qx - qn * ux, vy = qy - qn * uy, vz = qz - qn * uz;
        vxp[i] = (float)(-2.0 * k * vx);
        vyp[i] = (float)(-2.0 * k * vy);
        vzp[i] = (float)(-2.0 * k * vz);
        q2p[i] = FAST ? (float)inv2q : (float)(2.0 * qn);
        if (UNIFORM) {
            nqp[i] = (float)(2.0 * ((double)sv.unx * qx + (double)sv.uny * qy + (double)sv.unz * qz));
        } else {
            qxp[i] = (float)qx;
            qyp[i] = (float)qy;
            qzp[i] = (float)qz;
        }
        if (FOLD) {
            // The base phase enters the FP32 residual phase of every pair of
            // the chunk (|fr| <= 1/2 turn), so the chunk sums need no phasor.
            reinterpret_cast<float*>(st.phi)[i] = 6.28318530717958647692f * fr;
        } else {
            // |fr| <= 1/2 turn: the SFU sin/cos is accurate to ~5e-7 on [-pi, pi].
            const float kt = (float)sv.kt;
            float sp, cp;
            __sincosf(6.28318530717958647692f * fr, &sp, &cp);
            ws.ph[i][lane] = make_float2(-kt * sp, kt * cp);
        }
    }
}

// Unfolded variants, at every chunk boundary and at the item end: multiplies
// the lane's two-float chunk sums by the chunk phasor in FP64, adds them to
// the item's slots (tile-slot order) and clears the sums.
template <bool POL, class WS>
__device__ __forceinline__ void flush_chunk(const PrSolve& sv, int t, int g, int lane, WS& ws) {
    constexpr int NC = WS::kNC;
    const size_t slots = (size_t)sv.n_tiles * kPrTile;
    double* base = sv.partial + (size_t)g * 4 * slots;
#pragma unroll 2
    for (int i = 0; i < kPrPpl; ++i) {
        const size_t s = (size_t)t * kPrTile + lane + 32 * i;
        const float2 ph = ws.ph[i][lane];
        const double phr = ph.x, phi = ph.y;
        double v[4];
#pragma unroll
        for (int c = 0; c < (POL ? 2 : 4); ++c) {
            v[c] = (double)ws.hi[i * NC + c][lane] + (double)ws.lo[i * NC + c][lane];
            ws.hi[i * NC + c][lane] = 0.f;
            ws.lo[i * NC + c][lane] = 0.f;
        }
        // Each slot is updated by this one thread, in chunk order; the atomic
        // form only lets the warp go on without waiting for the loads.
        atomicAdd(base + 0 * slots + s, v[0] * phr - v[1] * phi);
        atomicAdd(base + 1 * slots + s, v[0] * phi + v[1] * phr);
        if (!POL) {
            atomicAdd(base + 2 * slots + s, v[2] * phr - v[3] * phi);
            atomicAdd(base + 3 * slots + s, v[2] * phi + v[3] * phr);
        }
    }
}

// Folded variants, once at the item end: multiplies the lane's two-float
// sums of the item by i k / (2 pi) in FP64 and adds them to the item's slots.
template <bool POL, class WS>
__device__ __forceinline__ void flush_item(const PrSolve& sv, int t, int g, int lane, WS& ws) {
    constexpr int NC = WS::kNC;
    const size_t slots = (size_t)sv.n_tiles * kPrTile;
    double* base = sv.partial + (size_t)g * 4 * slots;
    const double kt = sv.kt;
#pragma unroll 2
    for (int i = 0; i < kPrPpl; ++i) {
        const size_t s = (size_t)t * kPrTile + lane + 32 * i;
        double v[4];
#pragma unroll
        for (int c = 0; c < (POL ? 2 : 4); ++c)
            v[c] = (double)ws.hi[i * NC + c][lane] + (double)ws.lo[i * NC + c][lane];
        // Sub-items of one (group, tile) add into the same slots in sub
        // order (never two in one launch); the atomic form only lets the warp
        // go on without waiting for the loads.
        atomicAdd(base + 0 * slots + s, -kt * v[1]);
        atomicAdd(base + 1 * slots + s, kt * v[0]);
        if (!POL) {
            atomicAdd(base + 2 * slots + s, -kt * v[3]);
            atomicAdd(base + 3 * slots + s, kt * v[2]);
        }
    }
}

// Prepares the stage's rays for the item direction (lane j handles rays
// j, j+32).
// One-polarization kernels (POL) prepare the one amplitude column they sum;
// the unfolded ones (POLAR) keep it in polar form, e = {|a|, psi}, psi the
// amplitude's phase plus the ray phase -k u.rho, which the sweep adds to the
// pair's residual phase inside the FMA that forms it, so that a pair costs
// one multiply and two FMAs on the sums instead of a complex multiply-add.
// (In the folded kernels the same form measured 3x the field error and no
// faster; they keep the Cartesian amplitude.)
template <bool POL, bool POLAR, class WS>
__device__ __forceinline__ void prep_stage(PrRawRay* buf, int len, int lane, const PrSolve& sv,
                                           const WS& ws) {
    const double ux = ws.ux, uy = ws.uy, uz = ws.uz;
    for (int j = lane; j < len; j += 32) {
        const PrRawRay r = buf[j];
        double ur = ux * r.rx + uy * r.ry + uz * r.rz;
        double tx = r.rx - ur * ux, ty = r.ry - ur * uy, tz = r.rz - ur * uz;
        double perp2 = tx * tx + ty * ty + tz * tz;
        double turns = -sv.kt * ur;
        float f = (float)(turns - rint(turns));
        float sn = 0.f, cs = 1.f;
        if (!POLAR) __sincosf(6.28318530717958647692f * f, &sn, &cs);
        float rxf = (float)r.rx, ryf = (float)r.ry, rzf = (float)r.rz;
        float w = (float)(-2.0 * ur);
        float4 a = make_float4(rxf, ryf, rzf, (float)(sv.k * perp2));
        float4 b = make_float4(w, -2.f * (r.nx * rxf + r.ny * ryf + r.nz * rzf), r.nl, -w);
        float4 e;
        if (POLAR) {
            const float pr = sv.amp_src ? r.ep_re : r.es_re, pi = sv.amp_src ? r.ep_im : r.es_im;
            // |psi| <= 2 pi: f in [-1/2, 1/2] turns, atan2 in [-pi, pi].
            e = make_float4(hypotf(pr, pi), fmaf(6.28318530717958647692f, f, atan2f(pi, pr)),
                            0.f, 0.f);
        } else if (POL) {
            const float pr = sv.amp_src ? r.ep_re : r.es_re, pi = sv.amp_src ? r.ep_im : r.es_im;
            e = make_float4(pr * cs - pi * sn, pr * sn + pi * cs, 0.f, 0.f);
        } else {
            e = make_float4(r.es_re * cs - r.es_im * sn, r.es_re * sn + r.es_im * cs,
                            r.ep_re * cs - r.ep_im * sn, r.ep_re * sn + r.ep_im * cs);
        }
        float4 nn = make_float4(2.f * r.nx, 2.f * r.ny, 2.f * r.nz, 0.f);
        float4* o = reinterpret_cast<float4*>(buf + j);
        o[0] = a;
        o[1] = b;
        o[2] = e;
        o[3] = nn;
    }
}

// Adds the lane's FP32 partials into its two-float accumulators and clears
// them (every kFoldStages stages and at chunk and item ends).
// One-polarization kernels (POL) carry components 0 and 1 only.
template <bool POL, bool UNIFORM, class WS>
__device__ __forceinline__ void fold_acc(ScalarState<UNIFORM>& ls, WS& ws, int lane) {
    constexpr int NC = WS::kNC;
#pragma unroll
    for (int i = 0; i < kPrPpl; ++i)
#pragma unroll
        for (int c = 0; c < (POL ? 2 : 4); ++c) {
            float hi = ws.hi[i * NC + c][lane], lo = ws.lo[i * NC + c][lane];
            two_sum_acc(hi, lo, ls.acc[i][c]);
            ws.hi[i * NC + c][lane] = hi;
            ws.lo[i * NC + c][lane] = lo;
            ls.acc[i][c] = 0.f;
        }
}

template <bool POL, bool UNIFORM, class WS>
__device__ __forceinline__ void fold_acc(PackedState<UNIFORM>& ls, WS& ws, int lane) {
    constexpr int NC = WS::kNC;
#pragma unroll
    for (int i = 0; i < kPrPpl / 2; ++i)
#pragma unroll
        for (int c = 0; c < (POL ? 2 : 4); ++c) {
            const float2 v = ls.acc[i][c];
            float hi0 = ws.hi[(2 * i) * NC + c][lane], lo0 = ws.lo[(2 * i) * NC + c][lane];
            float hi1 = ws.hi[(2 * i + 1) * NC + c][lane], lo1 = ws.lo[(2 * i + 1) * NC + c][lane];
            two_sum_acc(hi0, lo0, v.x);
            two_sum_acc(hi1, lo1, v.y);
            ws.hi[(2 * i) * NC + c][lane] = hi0;
            ws.lo[(2 * i) * NC + c][lane] = lo0;
            ws.hi[(2 * i + 1) * NC + c][lane] = hi1;
            ws.lo[(2 * i + 1) * NC + c][lane] = lo1;
            ls.acc[i][c] = f2(0.f);
        }
}

template <bool UNIFORM>
__device__ __forceinline__ void clear_acc(ScalarState<UNIFORM>& ls) {
#pragma unroll
    for (int i = 0; i < kPrPpl; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) ls.acc[i][c] = 0.f;
}

template <bool UNIFORM>
__device__ __forceinline__ void clear_acc(PackedState<UNIFORM>& ls) {
#pragma unroll
    for (int i = 0; i < kPrPpl / 2; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) ls.acc[i][c] = f2(0.f);
}

// SFU sweep: one point per FP32 instruction, rcp.approx for the reciprocal
// (LIN does not apply).
template <bool UNIFORM, bool FOLD, bool POL, bool LIN, class WS>
__device__ __forceinline__ void sweep_stage(const PrRawRay* buf, int len, int lane,
                                            ScalarState<UNIFORM>& ls, WS& ws) {
    const float4* rec = reinterpret_cast<const float4*>(buf);
#pragma unroll 1
    for (int j = 0; j < len; ++j) {
        const float4 a = rec[4 * j + 0];
        const float4 b = rec[4 * j + 1];
        const float4 e = rec[4 * j + 2];
        float4 nn = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!UNIFORM) nn = rec[4 * j + 3];
#pragma unroll
        for (int i = 0; i < kPrPpl; ++i) {
            float num = fmaf(ls.vx[i], a.x, a.w);
            num = fmaf(ls.vy[i], a.y, num);
            num = fmaf(ls.vz[i], a.z, num);
            const float rd = rcp_approx(ls.q2[i] + b.x);
            // One column, unfolded: the amplitude's phase e.y joins the
            // residual phase inside the FMA that forms it.
            constexpr bool POLAR = POL && !FOLD;
            const float th = FOLD ? fmaf(num, rd, ls.phi[i]) : (POLAR ? fmaf(num, rd, e.y) : num * rd);
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
            if (POLAR) {
                const float m = amp * e.x;
                ls.acc[i][0] = fmaf(m, cs, ls.acc[i][0]);
                ls.acc[i][1] = fmaf(m, sn, ls.acc[i][1]);
                continue;
            }
            const float ac = amp * cs, as = amp * sn;
            ls.acc[i][0] = fmaf(e.x, ac, fmaf(-e.y, as, ls.acc[i][0]));
            ls.acc[i][1] = fmaf(e.x, as, fmaf(e.y, ac, ls.acc[i][1]));
            if (!POL) {
                ls.acc[i][2] = fmaf(e.z, ac, fmaf(-e.w, as, ls.acc[i][2]));
                ls.acc[i][3] = fmaf(e.z, as, fmaf(e.w, ac, ls.acc[i][3]));
            }
        }
    }
}

// Packed sweep: two points per f32x2 instruction, series reciprocal
// r0 (1 + e + e^2), or r0 (1 + e) when the planner bounds |e|^2 times the
// phase budget far below the tolerance (LIN: one f32x2 FMA fewer per pair of
// points).
template <bool UNIFORM, bool FOLD, bool POL, bool LIN, class WS>
__device__ __forceinline__ void sweep_stage(const PrRawRay* buf, int len, int lane,
                                            PackedState<UNIFORM>& ls, WS& ws) {
    constexpr int H = kPrPpl / 2;
    const float4* rec = reinterpret_cast<const float4*>(buf);
    // Two rays per iteration give the scheduler two independent sets of
    // chains (+3 % one-column, +1 % two-column on the far-field workload).
    // The folded (near-field) kernels switch chunks every few stages and ran
    // ~5 % slower unrolled; they and the general-normal two-column kernels,
    // which are at the register limit of three CTAs per SM, keep one.
#pragma unroll (((UNIFORM || POL) && !FOLD) ? 2 : 1)
    for (int j = 0; j < len; ++j) {
        const float4 a = rec[4 * j + 0];
        const float4 b = rec[4 * j + 1];
        const float4 e = rec[4 * j + 2];
        float4 nn = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!UNIFORM) nn = rec[4 * j + 3];
        const float2 ax = f2(a.x), ay = f2(a.y), az = f2(a.z), aw = f2(a.w);
        const float2 wn = f2(b.w), gg = f2(b.y), nl = f2(b.z);
        const float2 ex = f2(e.x), ey = f2(e.y), ez = f2(e.z), ew = f2(e.w);
        const float2 ney = f2(-e.y), new_ = f2(-e.w);
#pragma unroll
        for (int i = 0; i < H; ++i) {
            float2 num = __ffma2_rn(ls.vx[i], ax, aw);
            num = __ffma2_rn(ls.vy[i], ay, num);
            num = __ffma2_rn(ls.vz[i], az, num);
            // 1/(2|q| - 2u.rho) = r0 / (1 - e), e = 2u.rho r0 ~ r0 (1 + e + e^2)
            const float2 ep = __fmul2_rn(wn, ls.q2[i]);
            const float2 rd = LIN ? __ffma2_rn(ls.q2[i], ep, ls.q2[i])
                                  : __ffma2_rn(ls.q2[i], __ffma2_rn(ep, ep, ep), ls.q2[i]);
            constexpr bool POLAR = POL && !FOLD;
            const float2 th = FOLD ? __ffma2_rn(num, rd, ls.phi[i])
                                   : (POLAR ? __ffma2_rn(num, rd, ey) : __fmul2_rn(num, rd));
            float s0, c0, s1, c1;
            __sincosf(th.x, &s0, &c0);
            __sincosf(th.y, &s1, &c1);
            float2 gq;
            if (UNIFORM) {
                gq = __fadd2_rn(ls.nq[i], gg);
            } else {
                gq = __ffma2_rn(f2(nn.x), ls.qx[i],
                                __ffma2_rn(f2(nn.y), ls.qy[i], __ffma2_rn(f2(nn.z), ls.qz[i], gg)));
            }
            const float2 obl = __ffma2_rn(gq, rd, nl);
            const float2 amp = __fmul2_rn(obl, rd);
            if (POLAR) {
                const float2 m = __fmul2_rn(amp, ex);
                ls.acc[i][0] = __ffma2_rn(m, f2(c0, c1), ls.acc[i][0]);
                ls.acc[i][1] = __ffma2_rn(m, f2(s0, s1), ls.acc[i][1]);
                continue;
            }
            const float2 ac = __fmul2_rn(amp, f2(c0, c1));
            const float2 as = __fmul2_rn(amp, f2(s0, s1));
            ls.acc[i][0] = __ffma2_rn(ex, ac, __ffma2_rn(ney, as, ls.acc[i][0]));
            ls.acc[i][1] = __ffma2_rn(ex, as, __ffma2_rn(ey, ac, ls.acc[i][1]));
            if (!POL) {
                ls.acc[i][2] = __ffma2_rn(ez, ac, __ffma2_rn(new_, as, ls.acc[i][2]));
                ls.acc[i][3] = __ffma2_rn(ez, as, __ffma2_rn(ew, ac, ls.acc[i][3]));
            }
        }
    }
}

struct WarpPipe {
    PrRawRay* buf[2];
    uint64_t* bar[2];
    uint32_t phase;  // bit b: parity of the next completion of buffer b
};

// `extra` bytes beyond the copy are expected only by the stall test hook
// (PrCtl::stall_bytes); 0 otherwise.
__device__ __forceinline__ void issue_stage(WarpPipe& wp, int b, const PrRawRay* src, int len,
                                            int lane, uint32_t extra = 0) {
    if (lane == 0) {
        uint32_t bytes = (uint32_t)len * (uint32_t)sizeof(PrRawRay);
        mbar_arrive_expect_tx(wp.bar[b], bytes + extra);
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
template <bool UNIFORM, bool FAST, bool FOLD, bool POL, bool LIN>
__device__ bool process_item(const PrSolve& sv, long long local, WarpPipe& wp,
                             WarpSharedT<POL ? 2 : 4>& ws,
                             int lane, uint32_t wait_limit, uint32_t stall_bytes) {
    // local = (sub * groups + g) * n_tiles + t: sub-range `sub` of ray group g
    // against tile t. Sub-items of one (g, t) add into the same slots, so a
    // launch must never hold two of them (launches cover at most
    // groups * n_tiles consecutive items of a solve).
    const int t = (int)(local % sv.n_tiles);
    const long long rest = local / sv.n_tiles;
    const int g = sv.group_order[(int)(rest % sv.groups)];
    const int sub = (int)(rest / sv.groups);
    const long long n = sv.n_rays;
    const long long g0 = (long long)g * n / sv.groups;
    const long long g1 = (long long)(g + 1) * n / sv.groups;
    const int r0 = (int)(g0 + (g1 - g0) * sub / sv.subs);
    const int r1 = (int)(g0 + (g1 - g0) * (sub + 1) / sv.subs);
    if (r0 >= r1) return true;
    const int n_chunks = *sv.n_chunks_dev;
    const int* __restrict__ cb = sv.chunk_begin;

#pragma unroll
    for (int i = 0; i < kPrPpl * (POL ? 2 : 4); ++i) ws.hi[i][lane] = ws.lo[i][lane] = 0.f;

    using State = typename std::conditional<FAST, PackedState<UNIFORM>, ScalarState<UNIFORM>>::type;
    State st;
    clear_acc(st);
    int since_fold = 0;
    int cur_chunk = -1;
    int pos = r0;
    int c = chunk_of(cb, n_chunks, pos);
    int len = min(kPrStage, min(cb[c + 1], r1) - pos);
    int b = 0;
    issue_stage(wp, b, sv.recs + pos, len, lane, stall_bytes);
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
        const uint32_t par = (wp.phase >> b) & 1u;
        const bool ok = mbar_wait(wp.bar[b], par, wait_limit);
        wp.phase ^= (1u << b);
        if (!ok) {
            // Before the warp leaves, give both buffers' copies another
            // bounded wait, so that none is still writing into this warp's
            // shared memory when the block exits: this stage's (a slow copy
            // lands; a barrier that can never complete runs out again) and
            // the next stage's, already issued.
            mbar_wait(wp.bar[b], par, wait_limit);
            if (nlen > 0) {
                mbar_wait(wp.bar[b ^ 1], (wp.phase >> (b ^ 1)) & 1u, wait_limit);
                wp.phase ^= (1u << (b ^ 1));
            }
            return false;
        }
        if (c != cur_chunk) {
            if (!FOLD && cur_chunk >= 0) flush_chunk<POL>(sv, t, g, lane, ws);
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
            setup_points<UNIFORM, FAST, FOLD>(sv, t, lane, ws, st);
            cur_chunk = c;
        }
        prep_stage<POL, POL && !FOLD>(wp.buf[b], len, lane, sv, ws);
        __syncwarp();
        sweep_stage<UNIFORM, FOLD, POL, LIN>(wp.buf[b], len, lane, st, ws);
        // FP32 partials run over at most kFoldStages stages of one chunk.
        if (++since_fold == kFoldStages || nlen == 0 || nc != c) {
            fold_acc<POL>(st, ws, lane);
            since_fold = 0;
        }
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
    if (FOLD) flush_item<POL>(sv, t, g, lane, ws);
    else flush_chunk<POL>(sv, t, g, lane, ws);
    __syncwarp();
    return true;
}

// Every solve in `solves` must match the kernel's variant (normal mode and
// sweep); solves[s].item_begin is the prefix sum of the item counts in this
// launch, and the launch covers items [item_offset, item_offset + count) of
// each solve.
template <bool UNIFORM, bool FAST, bool FOLD, bool POL, bool LIN>
__global__ void __launch_bounds__(kPrWarpsPerCta * 32, (POL && !FOLD) ? 4 : 3)
pr_persistent_kernel(const PrSolve* __restrict__ solves, int n_solves, long long n_items,
                     unsigned long long* __restrict__ counter, int* __restrict__ err, PrCtl ctl) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    PrRawRay* bufs = reinterpret_cast<PrRawRay*>(smem) + warp * 2 * kPrStage;
    using WS = WarpSharedT<POL ? 2 : 4>;
    WS* wsh = reinterpret_cast<WS*>(smem + kPrWarpsPerCta * 2 * kPrStage * sizeof(PrRawRay)) + warp;
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
        int lo = 0, hi = n_solves - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (solves[mid].item_begin <= item) lo = mid;
            else hi = mid - 1;
        }
        const PrSolve& sv = solves[lo];
        const long long local = item - sv.item_begin + sv.item_offset;
        const bool ok = process_item<UNIFORM, FAST, FOLD, POL, LIN>(
            sv, local, wp, *wsh, lane, ctl.wait_limit, item == 0 ? ctl.stall_bytes : 0u);
        if (!ok) {
            if (lane == 0) atomicExch(err, 1);
            break;
        }
    }
}

// Dynamic shared memory of a launch: the warps' ray buffers and their state.
constexpr size_t pr_smem_bytes(bool pol) {
    return (size_t)kPrWarpsPerCta * 2 * kPrStage * sizeof(PrRawRay) +
           (size_t)kPrWarpsPerCta * (pol ? sizeof(WarpSharedT<2>) : sizeof(WarpSharedT<4>));
}

using PrKernel = void (*)(const PrSolve*, int, long long, unsigned long long*, int*, PrCtl);

// Kernel of a variant: bit 0 uniform normal, bit 1 packed sweep, bit 2 folded
// base phase, bit 3 one polarization, bit 4 linear series (PrPlan::variant();
// bit 4 only occurs with bit 1).
template <bool POL>
PrKernel pr_kernel_pol(int v) {
    static const PrKernel table[8] = {
        pr_persistent_kernel<false, false, false, POL, false>,
        pr_persistent_kernel<true, false, false, POL, false>,
        pr_persistent_kernel<false, true, false, POL, false>,
        pr_persistent_kernel<true, true, false, POL, false>,
        pr_persistent_kernel<false, false, true, POL, false>,
        pr_persistent_kernel<true, false, true, POL, false>,
        pr_persistent_kernel<false, true, true, POL, false>,
        pr_persistent_kernel<true, true, true, POL, false>};
    static const PrKernel lin[4] = {  // packed sweeps: uniform x folded
        pr_persistent_kernel<false, true, false, POL, true>,
        pr_persistent_kernel<true, true, false, POL, true>,
        pr_persistent_kernel<false, true, true, POL, true>,
        pr_persistent_kernel<true, true, true, POL, true>};
    if ((v & 16) && (v & 2)) return lin[(v & 1) | ((v >> 1) & 2)];
    return table[v & 7];
}

PrKernel pr_kernel(int variant) {
    return (variant & 8) ? pr_kernel_pol<true>(variant) : pr_kernel_pol<false>(variant);
}

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

// Per-solve planning scratch carved from the arena.
struct SolveBufs {
    double* sum;
    uint64_t *pk_in, *pk_out;
    int *pi_in, *pi_out;
    int* tile_perm;
    double *tpx, *tpy, *tpz, *tile_center;
    unsigned long long* amax;
    uint64_t *rk_in, *rk_out;
    int *ri_in, *ri_out, *flags, *run;
    int* chunk_begin;
    double* chunk_center;
    int* n_chunks;
    int* group_order;
    PrRawRay* recs;
    double* partial;
};

void carve(Arena& a, SolveBufs& b, int n, int m, int n_tiles, int groups, int sum_blocks) {
    const size_t slots = (size_t)n_tiles * kPrTile;
    b.sum = a.take<double>((size_t)sum_blocks * kSumFields);
    b.pk_in = a.take<uint64_t>(m);
    b.pk_out = a.take<uint64_t>(m);
    b.pi_in = a.take<int>(m);
    b.pi_out = a.take<int>(m);
    b.tile_perm = a.take<int>(slots);
    b.tpx = a.take<double>(slots);
    b.tpy = a.take<double>(slots);
    b.tpz = a.take<double>(slots);
    b.tile_center = a.take<double>(3 * (size_t)n_tiles);
    b.amax = a.take<unsigned long long>(1);
    b.rk_in = a.take<uint64_t>(n);
    b.rk_out = a.take<uint64_t>(n);
    b.ri_in = a.take<int>(n);
    b.ri_out = a.take<int>(n);
    b.flags = a.take<int>(n);
    b.run = a.take<int>(n);
    b.chunk_begin = a.take<int>((size_t)n + 1);
    b.chunk_center = a.take<double>(3 * (size_t)n);
    b.n_chunks = a.take<int>(1);
    b.group_order = a.take<int>(groups);
    b.recs = a.take<PrRawRay>(n);
    b.partial = a.take<double>((size_t)groups * 4 * slots);
}

struct HostSolveInfo {
    double f[kSumFields];
    double k = 0, d_lo = 0, rc[3], pc[3], rlo[3], rhi[3], plo[3], phi[3];
    Frame fr{};
};

// Pinned host area layout: [per-solve summaries][per-solve amax][per-solve
// n_chunks][error word][solve tables].
struct HostLayout {
    size_t sum_off, amax_off, nch_off, err_off, tab_off, total;
};

HostLayout host_layout(int count, int sum_blocks) {
    HostLayout L;
    size_t off = 0;
    L.sum_off = off;
    off = align_up(off + (size_t)count * sum_blocks * kSumFields * sizeof(double), 256);
    L.amax_off = off;
    off = align_up(off + (size_t)count * sizeof(double), 256);
    L.nch_off = off;
    off = align_up(off + (size_t)count * sizeof(int), 256);
    L.err_off = off;
    off = align_up(off + 64, 256);
    L.tab_off = off;
    off = align_up(off + (size_t)count * sizeof(PrSolve), 256);
    L.total = off;
    return L;
}

int sum_blocks_for(int num_sms) { return std::min(512, std::max(1, 2 * num_sms)); }

// Ray groups per tile: enough items to keep every resident warp busy, at
// least four stages of rays per item, partial slots within 1 GiB.
int plan_groups(int n, int m, int n_tiles, int num_sms, const PrOptions& opt) {
    if (opt.groups > 0) return std::min(opt.groups, kMaxGroups);
    long long ipw = opt.items_per_warp;
    if (opt.tune && opt.tune->use) opt.tune->find_ipw((size_t)n, (size_t)m, &ipw);
    long long want = (long long)num_sms * 12 * ipw;
    int g = (int)std::max<long long>(1, (want + n_tiles - 1) / n_tiles);
    g = std::min(g, std::max(1, n / (4 * kPrStage)));
    long long cap = (1LL << 30) / (32LL * n_tiles * kPrTile);
    g = (int)std::max<long long>(1, std::min<long long>(g, cap));
    return std::min(g, kMaxGroups);
}

}  // namespace

uint32_t PrTuneCache::size_key(size_t n, size_t m) {
    const int nb = n ? std::ilogb((double)n) : 0, mb = m ? std::ilogb((double)m) : 0;
    return (uint32_t)(nb & 0xff) << 8 | (uint32_t)(mb & 0xff);
}

uint64_t PrTuneCache::full_key(double energy_ev, double dist_mm, size_t n, size_t m) {
    const int eb = energy_ev > 0 ? (int)std::lround(std::log2(energy_ev)) : 0;
    const int db = dist_mm > 0 ? (int)std::lround(std::log2(dist_mm)) : 0;
    return (uint64_t)((eb + 128) & 0xff) << 24 | (uint64_t)((db + 128) & 0xff) << 16 |
           size_key(n, m);
}

void PrTuneCache::store(double energy_ev, double dist_mm, size_t n, size_t m, const PrTuned& t) {
    std::lock_guard<std::mutex> lock(mu);
    full[full_key(energy_ev, dist_mm, n, m)] = t;
    ipw[size_key(n, m)] = t.items_per_warp;
}

bool PrTuneCache::find(double energy_ev, double dist_mm, size_t n, size_t m, PrTuned* t) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = full.find(full_key(energy_ev, dist_mm, n, m));
    if (it == full.end()) return false;
    *t = it->second;
    return true;
}

bool PrTuneCache::find_ipw(size_t n, size_t m, long long* ipw_out) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = ipw.find(size_key(n, m));
    if (it == ipw.end()) return false;
    *ipw_out = it->second;
    return true;
}

size_t PrTuneCache::size() {
    std::lock_guard<std::mutex> lock(mu);
    return full.size();
}

void PrTuneCache::clear() {
    std::lock_guard<std::mutex> lock(mu);
    full.clear();
    ipw.clear();
}

const char* const kRouteReasons[kRouteReasonCount] = {
    "",
    "no rays",
    "rays of different energies",
    "non-positive energy",
    "ray and screen bounding boxes overlap",
    "no cell size meets the phase budget",
    "ray cell grid too fine",
    "non-finite ray or screen values",
    "amplitudes outside the FP32 range of the phase-reduced sums"};

Status PrWorkspace::ensure_host(size_t bytes) {
    if (bytes <= host_bytes) return Status::Ok();
    if (host_borrowed) return Status::Err(XK_ERR_OOM, "borrowed pinned area too small");
    if (host) cudaFreeHost(host);
    host = nullptr;
    host_bytes = 0;
    host_err = nullptr;
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
    if (host && !host_borrowed) cudaFreeHost(host);
    host = nullptr;
    host_bytes = 0;
    host_err = nullptr;
    host_borrowed = false;
}

size_t pr_plan_bytes(size_t n, size_t m, int num_sms, const PrOptions& opt) {
    if (n == 0 || m == 0) return 0;
    const int sum_blocks = sum_blocks_for(num_sms);
    const int n_tiles = (int)((m + kPrTile - 1) / kPrTile);
    const int g = plan_groups((int)n, (int)m, n_tiles, num_sms, opt);
    Arena a{nullptr, 0};
    SolveBufs b;
    carve(a, b, (int)n, (int)m, n_tiles, g, sum_blocks);
    // CUB radix sort of 64-bit keys + 32-bit values and the scan need at most
    // a few bytes per item; 16 per item plus 1 MiB bounds them.
    return a.off + 16 * std::max(n, m) + (1u << 20) + (2u << 20);
}

Status pr_plan(const PrSolveIn* in, int count, PrWorkspace& ws, cudaStream_t stream, int num_sms,
               const PrOptions& opt, std::vector<PrPlan>& plans, int* kernels,
               DevBuf* const* arenas) {
    plans.assign(count, PrPlan());
    int nk = 0;
    const int sum_blocks = sum_blocks_for(num_sms);
    std::vector<int> n_tiles(count, 0), groups(count, 0);
    size_t cub_need = 0;
    size_t need = 0;
    for (int s = 0; s < count; ++s) {
        PrPlan& P = plans[s];
        P.out = in[s].out;
        P.m = (int)in[s].m;
        if (in[s].n == 0 || in[s].m == 0) {
            P.routed = true;
            P.route_reason = 1;
            continue;
        }
        if (in[s].n > (size_t)INT32_MAX / 2 || in[s].m > (size_t)INT32_MAX / 2)
            return Status::Err(XK_ERR_INVALID, "too many rays or screen points for one solve");
        const int n = (int)in[s].n, m = (int)in[s].m;
        n_tiles[s] = (m + kPrTile - 1) / kPrTile;
        const int g = plan_groups(n, m, n_tiles[s], num_sms, opt);
        groups[s] = g;
        size_t c1 = 0, c2 = 0, c3 = 0;
        XK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, c1, (uint64_t*)nullptr,
                                                    (uint64_t*)nullptr, (int*)nullptr,
                                                    (int*)nullptr, n));
        XK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, c2, (uint64_t*)nullptr,
                                                    (uint64_t*)nullptr, (int*)nullptr,
                                                    (int*)nullptr, m));
        XK_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, c3, (int*)nullptr, (int*)nullptr, n));
        cub_need = std::max(cub_need, std::max(c1, std::max(c2, c3)));
        Arena a{nullptr, arenas ? 0 : need};
        SolveBufs b;
        carve(a, b, n, m, n_tiles[s], g, sum_blocks);
        if (arenas) XK_TRY(arenas[s]->ensure(a.off + 256));
        else need = a.off;
    }
    XK_TRY(ws.cub_tmp.ensure(cub_need + 256));
    if (!arenas) XK_TRY(ws.arena.ensure(need + 256));
    const HostLayout HL = host_layout(count, sum_blocks);
    XK_TRY(ws.ensure_host(HL.total));
    char* hbase = static_cast<char*>(ws.host);
    double* h_sum = reinterpret_cast<double*>(hbase + HL.sum_off);
    double* h_amax = reinterpret_cast<double*>(hbase + HL.amax_off);
    int* h_nch = reinterpret_cast<int*>(hbase + HL.nch_off);

    std::vector<SolveBufs> bufs(count);
    {
        size_t off = 0;
        for (int s = 0; s < count; ++s) {
            if (plans[s].routed) continue;
            Arena a{arenas ? arenas[s]->as<char>() : ws.arena.as<char>(), arenas ? 0 : off};
            carve(a, bufs[s], (int)in[s].n, (int)in[s].m, n_tiles[s], groups[s], sum_blocks);
            off = a.off;
        }
    }

    // --- A. summaries ------------------------------------------------------
    bool any = false;
    for (int s = 0; s < count; ++s) {
        if (plans[s].routed) continue;
        any = true;
        summary_kernel<<<sum_blocks, 256, 0, stream>>>(in[s].rays, (int)in[s].n, in[s].pix,
                                                        (int)in[s].m, bufs[s].sum);
        XK_CUDA_TRY(cudaGetLastError());
        XK_CUDA_TRY(cudaMemcpyAsync(h_sum + (size_t)s * sum_blocks * kSumFields, bufs[s].sum,
                                    (size_t)sum_blocks * kSumFields * sizeof(double),
                                    cudaMemcpyDeviceToHost, stream));
        ++nk;
    }
    if (!any) {
        if (kernels) *kernels += nk;
        return Status::Ok();
    }
    XK_CUDA_TRY(cudaStreamSynchronize(stream));

    std::vector<HostSolveInfo> info(count);
    for (int s = 0; s < count; ++s) {
        PrPlan& P = plans[s];
        if (P.routed) continue;
        HostSolveInfo& I = info[s];
        const double* hs = h_sum + (size_t)s * sum_blocks * kSumFields;
        for (int i = 0; i < kSumFields; ++i) {
            double v = hs[i];
            for (int bk = 1; bk < sum_blocks; ++bk) {
                double w = hs[bk * kSumFields + i];
                v = h_sum_ops[i] == 0 ? v + w : (h_sum_ops[i] == 1 ? std::min(v, w) : std::max(v, w));
            }
            I.f[i] = v;
        }
        const double* f = I.f;
        if (!(f[26] == 0.0)) {
            // NaN or infinite inputs: the FP64 sum propagates them the way
            // diffraction.rs:67-117 does; the planner's geometry would not.
            P.routed = true;
            P.route_reason = 7;
            continue;
        }
        if (f[32] > kF32AmpMax || (f[32] > 0.0 && f[32] < kF32AmpMin)) {
            P.routed = true;
            P.route_reason = 8;
            continue;
        }
        if (!(f[9] == f[10])) {
            P.routed = true;
            P.route_reason = 2;
            continue;
        }
        I.k = (f[9] / kChbar) * 1e7;
        if (!(I.k > 0) || !std::isfinite(I.k)) {
            P.routed = true;
            P.route_reason = 3;
            continue;
        }
        P.uniform_normal = f[11] == f[14] && f[12] == f[15] && f[13] == f[16];
        // One common polarization (es_j, ep_j) ~ (es_0, ep_0): sum A over
        // a_j = es_j, Ep = (ep_0 / es_0) A; with es_0 = 0 every es_j is 0 and
        // a_j = ep_j.
        const double a0r = f[28], a0i = f[29], b0r = f[30], b0i = f[31];
        const bool es0 = a0r != 0.0 || a0i != 0.0, ep0 = b0r != 0.0 || b0i != 0.0;
        P.one_pol = opt.polarization != 0 && f[27] <= kOnePolTol && (es0 || ep0);
        if (P.one_pol && es0) {
            // ep_0 / es_0 in extended precision (|es_0|^2 cannot underflow);
            // a ratio beyond FP64's range keeps both columns.
            const long double ar = a0r, ai = a0i, br = b0r, bi = b0i;
            const long double d = ar * ar + ai * ai;
            const double pr = (double)((br * ar + bi * ai) / d);
            const double pi = (double)((bi * ar - br * ai) / d);
            if (std::isfinite(pr) && std::isfinite(pi)) {
                P.dev.amp_src = 0;
                P.pol_es[0] = 1.0;
                P.pol_es[1] = 0.0;
                P.pol_ep[0] = pr;
                P.pol_ep[1] = pi;
            } else {
                P.one_pol = false;
            }
        } else if (P.one_pol) {
            P.dev.amp_src = 1;
            P.pol_es[0] = P.pol_es[1] = 0.0;
            P.pol_ep[0] = 1.0;
            P.pol_ep[1] = 0.0;
        }
        for (int a = 0; a < 3; ++a) {
            I.rlo[a] = f[3 + a];
            I.rhi[a] = f[6 + a];
            I.plo[a] = f[20 + a];
            I.phi[a] = f[23 + a];
            I.rc[a] = f[a] / (double)in[s].n;
            I.pc[a] = f[17 + a] / (double)in[s].m;
        }
        I.d_lo = box_distance(I.rlo, I.rhi, I.plo, I.phi);
        P.energy_ev = f[9];
        P.dist_mm = std::sqrt((I.pc[0] - I.rc[0]) * (I.pc[0] - I.rc[0]) +
                              (I.pc[1] - I.rc[1]) * (I.pc[1] - I.rc[1]) +
                              (I.pc[2] - I.rc[2]) * (I.pc[2] - I.rc[2]));
        if (!(I.d_lo > 0)) {
            P.routed = true;
            P.route_reason = 4;
            continue;
        }
        double u0[3] = {I.pc[0] - I.rc[0], I.pc[1] - I.rc[1], I.pc[2] - I.rc[2]};
        if (u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2] == 0) u0[2] = 1;
        normalize3(u0);
        double helper[3] = {std::fabs(u0[0]) < 0.9 ? 1.0 : 0.0, std::fabs(u0[0]) < 0.9 ? 0.0 : 1.0,
                            0.0};
        double dot = helper[0] * u0[0] + helper[1] * u0[1] + helper[2] * u0[2];
        double e1[3] = {helper[0] - dot * u0[0], helper[1] - dot * u0[1], helper[2] - dot * u0[2]};
        normalize3(e1);
        double e2[3] = {u0[1] * e1[2] - u0[2] * e1[1], u0[2] * e1[0] - u0[0] * e1[2],
                        u0[0] * e1[1] - u0[1] * e1[0]};
        for (int i = 0; i < 3; ++i) {
            I.fr.e1[i] = e1[i];
            I.fr.e2[i] = e2[i];
            I.fr.u0[i] = u0[i];
        }
    }

    // --- B. screen tiles ----------------------------------------------------
    any = false;
    for (int s = 0; s < count; ++s) {
        PrPlan& P = plans[s];
        if (P.routed) continue;
        any = true;
        HostSolveInfo& I = info[s];
        SolveBufs& B = bufs[s];
        const int m = (int)in[s].m;
        Frame pf = I.fr;
        pf.ox = I.pc[0];
        pf.oy = I.pc[1];
        pf.oz = I.pc[2];
        const double* axes[3] = {I.fr.e1, I.fr.e2, I.fr.u0};
        const double qmax[3] = {65535.0, 65535.0, 2097151.0};
        for (int ax = 0; ax < 3; ++ax) {
            double mn, mx;
            project_box(I.plo, I.phi, I.pc, axes[ax], &mn, &mx);
            pf.lo[ax] = mn;
            pf.scale[ax] = (mx > mn) ? qmax[ax] / (mx - mn) : 0.0;
        }
        pixel_keys_kernel<<<(m + 255) / 256, 256, 0, stream>>>(in[s].pix, m, pf, B.pk_in, B.pi_in);
        XK_CUDA_TRY(cudaGetLastError());
        size_t tmp = ws.cub_tmp.bytes;
        XK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp.ptr, tmp, B.pk_in, B.pk_out, B.pi_in,
                                                    B.pi_out, m, 0, 53, stream));
        XK_CUDA_TRY(cudaMemsetAsync(B.amax, 0, sizeof(unsigned long long), stream));
        tile_kernel<<<(n_tiles[s] * 32 + 255) / 256, 256, 0, stream>>>(
            in[s].pix, m, n_tiles[s], B.pi_out, B.tile_perm, B.tpx, B.tpy, B.tpz, B.tile_center,
            B.amax);
        XK_CUDA_TRY(cudaGetLastError());
        XK_CUDA_TRY(cudaMemcpyAsync(h_amax + s, B.amax, sizeof(double), cudaMemcpyDeviceToHost,
                                    stream));
        nk += 2;
    }
    if (any) XK_CUDA_TRY(cudaStreamSynchronize(stream));

    // --- C. ray chunks ------------------------------------------------------
    for (int s = 0; s < count; ++s) {
        PrPlan& P = plans[s];
        if (P.routed) continue;
        HostSolveInfo& I = info[s];
        SolveBufs& B = bufs[s];
        const int n = (int)in[s].n;
        const double a_max = h_amax[s] * 1.001;
        const double k = I.k;
        // Autotuned settings of this solve's bucket, if any.
        PrOptions o = opt;
        if (opt.tune && opt.tune->use) {
            PrTuned t;
            if (opt.tune->find(P.energy_ev, P.dist_mm, in[s].n, in[s].m, &t)) {
                o.phase_budget = std::min(t.phase_budget, opt.phase_budget);
                o.sweep = t.sweep;
                P.tuned = true;
            }
        }
        CellGrid cg{};
        cg.fr = I.fr;
        cg.fr.ox = I.rc[0];
        cg.fr.oy = I.rc[1];
        cg.fr.oz = I.rc[2];
        double ext[3];
        const double* axes[3] = {I.fr.e1, I.fr.e2, I.fr.u0};
        for (int ax = 0; ax < 3; ++ax) {
            double mn, mx;
            project_box(I.rlo, I.rhi, I.rc, axes[ax], &mn, &mx);
            cg.fr.lo[ax] = mn;
            ext[ax] = mx - mn;
        }
        auto cell_radius = [&](double h, double cell[3]) {
            double sq = 0;
            for (int ax = 0; ax < 3; ++ax) {
                cell[ax] = ext[ax] <= h ? ext[ax] : h;
                sq += 0.25 * cell[ax] * cell[ax];
            }
            return std::sqrt(sq);
        };
        double cell[3];
        const double budget = effective_phase_budget(o);
        double h_hi = 2.0 * std::max(ext[0], std::max(ext[1], ext[2])) + 1e-300;
        double h_lo = 0.0;
        if (phase_bound(k, a_max, cell_radius(h_hi, cell), I.d_lo) <= budget) {
            h_lo = h_hi;
        } else {
            for (int it = 0; it < 200; ++it) {
                double h = 0.5 * (h_lo + h_hi);
                if (phase_bound(k, a_max, cell_radius(h, cell), I.d_lo) <= budget) h_lo = h;
                else h_hi = h;
            }
        }
        const double h = h_lo;
        const double b_max = cell_radius(h, cell);
        if (!(h > 0)) {
            P.routed = true;
            P.route_reason = 5;
            continue;
        }
        bool too_fine = false;
        for (int ax = 0; ax < 3; ++ax) {
            cg.cell[ax] = cell[ax];
            double cnt = cell[ax] > 0 ? std::floor(ext[ax] / cell[ax]) + 1.0 : 1.0;
            if (cnt > 2097151.0) too_fine = true;
            cg.n[ax] = (long long)cnt;
        }
        if (too_fine) {
            P.routed = true;
            P.route_reason = 6;
            continue;
        }
        {
            // 2^E bounds every screen and ray coordinate; multiples of 2^(E-52)
            // then subtract from any screen coordinate exactly.
            double amax = 0.0;
            for (int a = 0; a < 3; ++a)
                amax = std::max(amax, std::max(std::max(std::fabs(I.plo[a]), std::fabs(I.phi[a])),
                                               std::max(std::fabs(I.rlo[a]), std::fabs(I.rhi[a]))));
            const int e = amax > 0 ? std::ilogb(amax) + 2 : -1000;
            cg.quantum = std::ldexp(1.0, e - 52);
            cg.inv_quantum = std::ldexp(1.0, 52 - e);
        }
        P.phase_bound = phase_bound(k, a_max, b_max, I.d_lo);
        // |e| = |u.rho| / |q| <= b / (d_lo - b): the series reciprocal's
        // argument.
        P.rcp_bound = b_max / std::max(I.d_lo - b_max, 1e-300);
        P.fast = o.sweep >= 1 || (o.sweep < 0 && P.rcp_bound <= kSeriesRcpBound);
        // The linear series drops r0 e^2: a relative error of at most e^2 in
        // the reciprocal, |residual phase| e^2 in the phase (a bias shared by
        // all pairs). Used where that stays below a tenth of the tolerance.
        P.lin = P.fast && (o.sweep == 2 ||
                           (o.sweep < 0 &&
                            P.rcp_bound * P.rcp_bound * budget <= 0.1 * o.tolerance));
        {
            // Fold the base phase into the sweep when ray groups span many
            // chunks and chunks hold few rays (near field): per-chunk set-up
            // and flushes then disappear, at the price of a phase add per
            // pair in the sweep. Non-empty cells bound the chunk count from
            // above.
            double cells = 1.0;
            for (int ax = 0; ax < 3; ++ax) cells *= (double)cg.n[ax];
            const double est_chunks = std::min(cells, (double)n);
            P.fold = est_chunks >= kFoldChunksPerGroup * (double)groups[s] &&
                     (double)n < kFoldRaysPerChunk * est_chunks;
        }

        ray_keys_kernel<<<(n + 255) / 256, 256, 0, stream>>>(in[s].rays, n, cg, B.rk_in, B.ri_in);
        XK_CUDA_TRY(cudaGetLastError());
        size_t tmp = ws.cub_tmp.bytes;
        XK_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp.ptr, tmp, B.rk_in, B.rk_out, B.ri_in,
                                                    B.ri_out, n, 0, 63, stream));
        head_flags_kernel<<<(n + 255) / 256, 256, 0, stream>>>(B.rk_out, n, B.flags);
        XK_CUDA_TRY(cudaGetLastError());
        tmp = ws.cub_tmp.bytes;
        XK_CUDA_TRY(cub::DeviceScan::InclusiveSum(ws.cub_tmp.ptr, tmp, B.flags, B.run, n, stream));
        chunk_table_kernel<<<(n + 255) / 256, 256, 0, stream>>>(B.rk_out, B.flags, B.run, n, cg,
                                                                 B.chunk_begin, B.chunk_center,
                                                                 B.n_chunks);
        XK_CUDA_TRY(cudaGetLastError());
        records_kernel<<<(n + 255) / 256, 256, 0, stream>>>(in[s].rays, n, B.ri_out, B.run,
                                                             B.chunk_center, B.recs);
        XK_CUDA_TRY(cudaGetLastError());
        group_order_kernel<<<1, 1024, 0, stream>>>(B.chunk_begin, B.n_chunks, n, groups[s],
                                                   B.group_order);
        XK_CUDA_TRY(cudaGetLastError());
        nk += 6;

        PrSolve& D = P.dev;
        D.recs = B.recs;
        D.chunk_begin = B.chunk_begin;
        D.chunk_center = B.chunk_center;
        D.n_chunks_dev = B.n_chunks;
        D.tpx = B.tpx;
        D.tpy = B.tpy;
        D.tpz = B.tpz;
        D.tile_center = B.tile_center;
        D.group_order = B.group_order;
        D.partial = B.partial;
        D.item_begin = 0;
        D.item_offset = 0;
        D.subs = 1;
        D.n_items = (long long)n_tiles[s] * groups[s];
        D.n_rays = n;
        D.n_tiles = n_tiles[s];
        D.groups = groups[s];
        D.k = k;
        {
            // k/(2 pi) as a double-double, k taken as the FP64 value the
            // reference computes (E / CHBAR * 1e7).
            const long double kt_ld = (long double)k / (2.0L * 3.14159265358979323846264338327950288L);
            D.kt = (double)kt_ld;
            D.kt_lo = (double)(kt_ld - (long double)D.kt);
        }
        D.unx = (float)I.f[11];
        D.uny = (float)I.f[12];
        D.unz = (float)I.f[13];
        P.tile_perm = B.tile_perm;
        P.n_tiles = n_tiles[s];
        P.groups = groups[s];
        P.n_chunks_host = h_nch + s;
        *P.n_chunks_host = 0;
    }
    if (kernels) *kernels += nk;
    return Status::Ok();
}

Status pr_zero_partials(const PrPlan& P, cudaStream_t stream) {
    const size_t slots = (size_t)P.n_tiles * kPrTile;
    XK_CUDA_TRY(cudaMemsetAsync(P.dev.partial, 0, (size_t)P.groups * 4 * slots * sizeof(double),
                                stream));
    return Status::Ok();
}

Status pr_launch(const PrSolve* d_table, int n_solves, long long n_items, int variant,
                 unsigned long long* d_counter, int* d_err, cudaStream_t stream, int num_sms,
                 int max_ctas_per_sm, const PrCtl& ctl) {
    if (n_items <= 0) return Status::Ok();
    PrKernel kern = pr_kernel(variant);
    const size_t smem = pr_smem_bytes((variant & 8) != 0);
    XK_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    XK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPrWarpsPerCta * 32,
                                                              smem));
    per_sm = std::max(per_sm, 1);
    if (max_ctas_per_sm > 0) per_sm = std::min(per_sm, max_ctas_per_sm);
    long long grid = (long long)num_sms * per_sm;
    grid = std::max<long long>(1, std::min(grid, (n_items + kPrWarpsPerCta - 1) / kPrWarpsPerCta));
    kern<<<(unsigned)grid, kPrWarpsPerCta * 32, smem, stream>>>(d_table, n_solves, n_items,
                                                                d_counter, d_err, ctl);
    XK_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

Status pr_finalize(const PrPlan& P, cudaStream_t stream) {
    const int slots = P.n_tiles * kPrTile;
    finalize_kernel<<<(slots + 255) / 256, 256, 0, stream>>>(
        P.dev.partial, P.tile_perm, P.groups, slots, P.out, P.one_pol ? 1 : 0,
        make_double2(P.pol_es[0], P.pol_es[1]), make_double2(P.pol_ep[0], P.pol_ep[1]));
    XK_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

Status pr_reserve_plan_host(PrWorkspace& ws, int count, int num_sms) {
    return ws.ensure_host(host_layout(count, sum_blocks_for(num_sms)).total);
}

Status pr_reserve_exec(PrWorkspace& ws, int count, int num_sms) {
    const HostLayout HL = host_layout(count, sum_blocks_for(num_sms));
    XK_TRY(ws.ensure_host(HL.total));
    XK_TRY(ws.solves.ensure(std::max<size_t>(1, count) * sizeof(PrSolve)));
    XK_TRY(ws.ctrl.ensure(kPrCtrlBytes));
    if (!ws.ev[0]) XK_CUDA_TRY(cudaEventCreate(&ws.ev[0]));
    if (!ws.ev[1]) XK_CUDA_TRY(cudaEventCreate(&ws.ev[1]));
    return Status::Ok();
}

Status pr_execute_enqueue(std::vector<PrPlan>& plans, PrWorkspace& ws, cudaStream_t stream,
                          int num_sms, bool time_kernels, PrExecReport* rep) {
    PrExecReport local;
    PrExecReport& R = rep ? *rep : local;
    const int count = (int)plans.size();
    const HostLayout HL = host_layout(count, sum_blocks_for(num_sms));
    XK_TRY(pr_reserve_exec(ws, count, num_sms));
    char* hbase = static_cast<char*>(ws.host);
    PrSolve* h_tab = reinterpret_cast<PrSolve*>(hbase + HL.tab_off);
    int* h_nch = reinterpret_cast<int*>(hbase + HL.nch_off);
    ws.host_err = reinterpret_cast<int*>(hbase + HL.err_off);
    *ws.host_err = 0;
    unsigned long long* d_counters = reinterpret_cast<unsigned long long*>(ws.ctrl.ptr);
    int* d_err = reinterpret_cast<int*>(static_cast<char*>(ws.ctrl.ptr) + kPrCtrlErrOffset);
    XK_CUDA_TRY(cudaMemsetAsync(ws.ctrl.ptr, 0, kPrCtrlBytes, stream));

    // Group the planned solves by kernel variant into contiguous tables.
    struct Launch {
        int first, count;
        long long items;
        int variant;
    };
    std::vector<Launch> launches;
    int tab = 0;
    for (int variant = 0; variant < kPrVariants; ++variant) {
        Launch L{tab, 0, 0, variant};
        for (int s = 0; s < count; ++s) {
            PrPlan& P = plans[s];
            if (P.routed || P.variant() != variant) continue;
            P.dev.item_begin = L.items;
            h_tab[tab++] = P.dev;
            L.items += P.dev.n_items;
            L.count++;
            XK_TRY(pr_zero_partials(P, stream));
        }
        if (L.count) launches.push_back(L);
    }
    if (tab == 0) return Status::Ok();
    XK_CUDA_TRY(cudaMemcpyAsync(ws.solves.ptr, h_tab, (size_t)tab * sizeof(PrSolve),
                                cudaMemcpyHostToDevice, stream));
    if (time_kernels) XK_CUDA_TRY(cudaEventRecord(ws.ev[0], stream));
    int li = 0;
    PrCtl ctl = ws.ctl;
    ws.ctl.stall_bytes = 0;  // the stall test hook arms one execution only
    for (const Launch& L : launches) {
        XK_TRY(pr_launch(reinterpret_cast<const PrSolve*>(ws.solves.ptr) + L.first, L.count,
                         L.items, L.variant, d_counters + li, d_err, stream, num_sms, 0, ctl));
        ctl.stall_bytes = 0;
        R.kernels += 1;
        R.n_items += L.items;
        ++li;
    }
    if (time_kernels) XK_CUDA_TRY(cudaEventRecord(ws.ev[1], stream));
    for (int s = 0; s < count; ++s) {
        PrPlan& P = plans[s];
        if (P.routed) continue;
        XK_TRY(pr_finalize(P, stream));
        XK_CUDA_TRY(cudaMemcpyAsync(h_nch + s, P.dev.n_chunks_dev, sizeof(int),
                                    cudaMemcpyDeviceToHost, stream));
        R.kernels += 1;
    }
    XK_CUDA_TRY(cudaMemcpyAsync(ws.host_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    return Status::Ok();
}

Status pr_execute_finish(std::vector<PrPlan>& plans, PrWorkspace& ws, PrExecReport* rep) {
    if (rep && rep->kernels > 0 && ws.ev[0]) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ws.ev[0], ws.ev[1]) == cudaSuccess) rep->main_kernel_ms = ms;
    }
    for (auto& P : plans)
        if (!P.routed && P.n_chunks_host) P.n_chunks = *P.n_chunks_host;
    if (ws.host_err && *ws.host_err != 0)
        return Status::Err(XK_ERR_TIMEOUT, "persistent kernel: a bounded wait for a ray stage ran out");
    return Status::Ok();
}

}  // namespace xk
