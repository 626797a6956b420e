// 2-D Fresnel propagation (waves::fresnel::fresnel_propagate,
// src/waves/fresnel.rs:53-106) on B200:
//
//   U(x_ix, z_iz) = sum_j es_j exp(i a ((x_ix - x_j)^2 + (z_iz - z_j)^2)),  a = k / (2 d)
//
// over a regular nx x nz screen (index iz * nx + ix), k = E / CHBAR * 1e7.
//
// Two paths:
//
// * XK_PATH_F64: the reference's sum run directly in FP64, one thread per
//   screen point, rays staged through shared memory, the per-term operations
//   in the reference's order (explicitly rounded, no FMA contraction) and the
//   terms added in ray order.
//
// * XK_PATH_SEPARABLE: on a regular screen the Fresnel kernel factorises,
//       exp(i a r^2) = exp(i a (x_ix - x_j)^2) * exp(i a (z_iz - z_j)^2),
//   so U = Z diag(es) X^T is a complex matrix product with the ray index as
//   the contraction. As a real product with interleaved (re, im) columns,
//       C[iz][n(ix, c)] = sum_k A[iz][k] B[n(ix, c)][k],
//       A[iz][2j] = Re Z, A[iz][2j+1] = Im Z,
//       B[n(ix,0)][2j] = Re W, B[n(ix,0)][2j+1] = -Im W, B[n(ix,1)][2j] = Im W, B[n(ix,1)][2j+1] = Re W,
//   with W = es X / max|es| and, per 128-point block of x, the real parts in
//   its first 128 columns and the imaginary parts in the next 128:
//   n(ix, c) = 256 (ix / 128) + 128 c + ix % 128. One fused kernel computes
//   it on the tensor cores without ever writing A or B to memory: per block
//   of 32 rays, a stager warp writes the rays' split coordinates to a ring of
//   shared-memory buffers, eight producer warps form the CTA's A (128 z rows)
//   and B (128 x points, 256 rows) tiles from them, split each phasor into
//   f16 hi + lo parts and store them in shared memory in the
//   128-byte-swizzled K-major layout; one thread issues tcgen05.mma kind::f16 (f32 accumulation in tensor
//   memory) for A_hi B_hi + A_hi B_lo + A_lo B_hi, which keeps ~2^-21 of each
//   phasor; four epilogue warps drain the accumulator into an FP64 partial
//   every kFSeg ray blocks (the tensor cores' f32 accumulation error grows
//   with the number of accumulated blocks), alternating between two TMEM
//   accumulators so that draining overlaps the next segment. K-split partials
//   are added in FP64 in split order (results do not depend on scheduling).

#include <cuda_fp16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>

#include "xk_ctx.cuh"
#include "xk_sm100.cuh"

namespace xk {
namespace {

constexpr double kInv2Pi = 0.15915494309189533577;

// ---- shared pieces -----------------------------------------------------------

// x_i = lo + (hi - lo) * i / max(n - 1, 1), evaluated as the reference does
// (src/waves/fresnel.rs:70-75).
__global__ void coords_kernel(double lo, double hi, size_t n, double* __restrict__ out) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double den = (double)(n > 1 ? n - 1 : 1);
    out[i] = __dadd_rn(lo, __ddiv_rn(__dmul_rn(__dsub_rn(hi, lo), (double)i), den));
}

// ---- FP64 direct sum ---------------------------------------------------------

constexpr int kF64Threads = 256;

__global__ void __launch_bounds__(kF64Threads)
fresnel_f64_kernel(const double* __restrict__ rx, const double* __restrict__ rz,
                   const double* __restrict__ er, const double* __restrict__ ei, size_t n,
                   const double* __restrict__ xp, const double* __restrict__ zp, size_t nx,
                   size_t total, double pre, double* __restrict__ o_re, double* __restrict__ o_im) {
    __shared__ double sx[kF64Threads], sz[kF64Threads], sr[kF64Threads], si[kF64Threads];
    const size_t idx = blockIdx.x * (size_t)kF64Threads + threadIdx.x;
    const bool valid = idx < total;
    const size_t iz = valid ? idx / nx : 0, ix = valid ? idx - iz * nx : 0;
    const double px = valid ? xp[ix] : 0.0, pz = valid ? zp[iz] : 0.0;
    double s_re = 0.0, s_im = 0.0;
    for (size_t base = 0; base < n; base += kF64Threads) {
        const size_t j = base + threadIdx.x;
        if (j < n) {
            sx[threadIdx.x] = rx[j];
            sz[threadIdx.x] = rz[j];
            sr[threadIdx.x] = er[j];
            si[threadIdx.x] = ei[j];
        }
        __syncthreads();
        const int len = (int)min((size_t)kF64Threads, n - base);
        for (int t = 0; t < len; ++t) {
            // dx, dz, r2 = dx*dx + dz*dz, phase = (0, pre) * r2, exp of it,
            // es * phasor, sum += (src/waves/fresnel.rs:87-94).
            const double dx = __dsub_rn(px, sx[t]);
            const double dz = __dsub_rn(pz, sz[t]);
            const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dz, dz));
            double sn, cs;
            sincos(__dmul_rn(pre, r2), &sn, &cs);
            const double a = sr[t], b = si[t];
            s_re = __dadd_rn(s_re, __dsub_rn(__dmul_rn(a, cs), __dmul_rn(b, sn)));
            s_im = __dadd_rn(s_im, __dadd_rn(__dmul_rn(a, sn), __dmul_rn(b, cs)));
        }
        __syncthreads();
    }
    if (valid) {
        o_re[idx] = s_re;
        o_im[idx] = s_im;
    }
}

// ---- fused separable product on the tensor cores --------------------------------

constexpr int kFRays = 32;                       // rays per block: K = 64 halves (re, im)
constexpr int kFStages = 2;
constexpr uint32_t kFA = 128 * 64 * 2;           // one A tile (hi or lo): 128 rows x 128 B
constexpr uint32_t kFB = 256 * 64 * 2;           // one B tile: 256 rows x 128 B
constexpr uint32_t kFStage = 2 * kFA + 2 * kFB;  // A_hi | A_lo | B_hi | B_lo
constexpr int kFEpiThreads = 128;                // warps 1..4
#ifndef XK_FRESNEL_PROD_WARPS
#define XK_FRESNEL_PROD_WARPS 8
#endif
#ifndef XK_FRESNEL_ROWS_PER
#define XK_FRESNEL_ROWS_PER 2
#endif
constexpr int kFProdThreads = 32 * XK_FRESNEL_PROD_WARPS;  // warps 5..
constexpr int kFRowsPer = XK_FRESNEL_ROWS_PER;             // A rows (and x points) per producer
constexpr int kFRowThreads = 128 / kFRowsPer;              // producers per ray group
constexpr int kFChunks = 8 / (kFProdThreads / kFRowThreads);  // 16-byte chunks per producer
static_assert(kFChunks * (kFProdThreads / kFRowThreads) == 8 && kFRowThreads % 32 == 0,
              "producers must tile the 128 rows x 8 chunks of a block");
constexpr int kFThreads = 32 + kFEpiThreads + kFProdThreads + 32;  // + the ray stager warp
constexpr int kFRayBufs = 4;  // staged ray blocks in flight
constexpr int kFSeg = 20;                        // ray blocks (60 K blocks) per f32 segment
// Polls of the issuer's final wait for its MMAs (never fewer, whatever the
// caller's wait limit): the accumulators are freed after it.
constexpr uint32_t kMmaDrainPolls = 1u << 22;
constexpr int kFN = 256;                         // accumulator columns (N of the UMMA)
// Ray staging (one block per ring buffer), per ray 8 floats: {z hi, x hi,
// z lo, x lo} and {frac(a z^2), frac(a x^2), es_re, es_im} (coordinates
// relative to the screen centre, amplitude scaled by 1 / max|es|).
constexpr uint32_t kFRayBytes = kFRays * 32;
// Epilogue staging: per epilogue warp 32 rows of 16 FP64 values, rows 144
// bytes apart (16-byte stores of 32 lanes then meet all banks once).
constexpr uint32_t kFEpiRow = 144;
constexpr uint32_t kFEpiBytes = 4 * 32 * kFEpiRow;
constexpr size_t kFSmem = 1024 + (size_t)kFStages * kFStage + kFRayBufs * kFRayBytes + kFEpiBytes + 256;

struct FusedArgs {
    const double *rx, *rz, *er, *ei;
    size_t n;
    int ray_blocks, splits;
    const double *xp, *zp;
    size_t nx, nz;
    double a_turns;    // k / (2 d) / (2 pi)
    double inv_scale;  // 1 / max|es|
    double ox, oz;     // origin of the phase split (screen centre)
    double* partial;   // [splits][m_pad][n_pad]
    int m_pad, n_pad;
    int* err;
    uint32_t wait_limit;  // polls of every bounded mbarrier wait
    uint32_t stall;       // test hook: extra arrivals stage 0's barrier waits for (never made)
};

// Byte offset of 16-byte chunk c (0..7) of row r in a 128-byte-swizzled tile.
__device__ __forceinline__ uint32_t sw128(uint32_t r, uint32_t c) {
    return r * 128u + ((c ^ (r & 7u)) << 4);
}

// Phase split. With p, r relative to the screen centre the phase in turns is
//     t = a (p - r)^2 = P(p) + kappa(p) r + R(r),
//     P = frac(a p^2), R = frac(a r^2), kappa = -2 a p,
// where P and R are reduced in FP64 once per screen row and per ray. The
// cross term kappa r (up to 2^21 turns, checked on the host) is formed
// exactly in FP32 from hi/lo splits of kappa and r: the rounded product
// kh*rh, its FMA error term, and the two small cross products; its integer
// part drops out and the fractional remainder keeps ~1e-7 turn.
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: (x + kMagic) - kMagic = rint(x), |x| < 2^22

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// The same for a row of A (.x) and a row of B (.y) at once on sm_100's packed
// f32x2 instructions, with the operation sequence and roundings of the scalar
// form: p1 = kh rh rounded, e1 = its FMA error, f1 = p1 - rint(p1),
// t = (pr + f1) + (kh rl + kl rh + e1), result t - rint(t). rint is the
// magic-number rounding (exact and sign-symmetric for |x| < 2^22), and the
// product is carried negated (khn = -kh) so that every step is one packed
// FMA, multiply or add; a - b is formed as fma(b, -1, a).
__device__ __forceinline__ float2 pair_turns2(float2 kh, float2 khn, float2 kl, float2 pr,
                                              float2 rh, float2 rl) {
    const float2 m = f2(kMagic), mn = f2(-kMagic), one_n = f2(-1.f);
    const float2 p1n = __fmul2_rn(khn, rh);                          // -p1
    const float2 e1 = __ffma2_rn(kh, rh, p1n);                       // kh rh - p1
    const float2 r1 = __fadd2_rn(__fadd2_rn(p1n, m), mn);            // rint(-p1)
    const float2 f1n = __ffma2_rn(r1, one_n, p1n);                   // -f1
    float2 sm = __ffma2_rn(kh, rl, e1);
    sm = __ffma2_rn(kl, rh, sm);
    const float2 t = __fadd2_rn(__ffma2_rn(f1n, one_n, pr), sm);    // (pr + f1) + sm
    const float2 rt = __fadd2_rn(__fadd2_rn(t, m), mn);
    return __ffma2_rn(rt, one_n, t);                                 // t - rint(t)
}

// hi/lo float split of a double and frac(a v^2) as a float.
__device__ __forceinline__ void split_coord(double v, double a, float* hi, float* lo, float* fr) {
    *hi = (float)v;
    *lo = (float)(v - (double)*hi);
    const double t = (a * v) * v;
    *fr = (float)(t - rint(t));
}

// (a, b) -> f16x2 hi (round to nearest) and f16x2 lo = (a, b) - hi.
__device__ __forceinline__ void split16x2(float a, float b, uint32_t* hi, uint32_t* lo) {
    const __half2 h = __floats2half2_rn(a, b);
    const float2 back = __half22float2(h);
    const float2 d = __ffma2_rn(back, f2(-1.f), make_float2(a, b));
    const __half2 l = __floats2half2_rn(d.x, d.y);
    *hi = *reinterpret_cast<const uint32_t*>(&h);
    *lo = *reinterpret_cast<const uint32_t*>(&l);
}

// (a + ib)(c + is) with explicit roundings, so that every kernel variant forms
// the same W bit for bit (no compiler-chosen FMA contraction).
__device__ __forceinline__ float cmul_re(float a, float b, float c, float s) {
    return __fmaf_rn(a, c, __fmul_rn(-b, s));
}
__device__ __forceinline__ float cmul_im(float a, float b, float c, float s) {
    return __fmaf_rn(a, s, __fmul_rn(b, c));
}

// (x, y) -> (x, -y) and (y, x) on packed f16 pairs (sign flip, half swap).
__device__ __forceinline__ uint32_t neg_hi(uint32_t v) { return v ^ 0x80000000u; }
__device__ __forceinline__ uint32_t swap_halves(uint32_t v) { return __byte_perm(v, 0, 0x1032); }

// Epilogue role (warps 1..4): drains each finished accumulator segment into
// this CTA's 128 rows of the FP64 split partial; `arrive_empty(b)` releases
// accumulator b to the MMA issuer. Warp w reads TMEM lanes 32 (w % 4) .. + 31
// (rows qd*32 .. +31 of the tile); lane l owns row qd*32 + l. Per 16-column
// chunk the lane converts its values to FP64 in its shared-memory staging row
// and hands the row to a bulk copy: the first segment stores it, later ones
// add it to the partial at the memory side (FP64 add, round to nearest). A
// segment's operations complete before the next segment's start, so the
// partial is s0 + s1 + ... in segment order, independent of timing. `stage`:
// this warp's 32 staging rows.
template <class ArriveEmpty>
__device__ __forceinline__ void drain_role(const FusedArgs& g, int warp, int lane, int mt, int nt,
                                           int sp, int nseg, uint32_t tmem, uint64_t* acc_full,
                                           unsigned char* stage, volatile int* flag,
                                           ArriveEmpty arrive_empty) {
    using namespace sm100;
    const int qd = warp & 3;
    if (nseg == 0) {
        double* rows0 = g.partial + ((size_t)sp * g.m_pad + (size_t)mt * 128 + qd * 32) * g.n_pad +
                        (size_t)nt * kFN + lane;
        for (int rr = 0; rr < 32; ++rr)
            for (int c = 0; c < kFN; c += 32) rows0[(size_t)rr * g.n_pad + c] = 0.0;
        return;
    }
    double* grow = g.partial + ((size_t)sp * g.m_pad + (size_t)mt * 128 + qd * 32 + lane) * g.n_pad +
                   (size_t)nt * kFN;
    unsigned char* srow = stage + lane * kFEpiRow;
    const uint32_t s_addr = smem_u32(srow);
    for (int q = 0; q < nseg; ++q) {
        const int b = q & 1;
        const bool ok = mbar_wait(&acc_full[b], (uint32_t)(q >> 1) & 1u, g.wait_limit);
        if (!__all_sync(0xffffffffu, ok)) {
            *flag = 1;
            break;
        }
        tc_fence_after();
        bulk_wait_all();  // the previous segment's writes to these rows are performed
#pragma unroll 1
        for (int c = 0; c < kFN / 16; ++c) {
            float v[16];
            tmem_ld_16cols(tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(b * kFN + c * 16), v);
            bulk_wait_read();  // the staging row is free again
#pragma unroll
            for (int k = 0; k < 8; ++k)
                reinterpret_cast<double2*>(srow)[k] =
                    make_double2((double)v[2 * k], (double)v[2 * k + 1]);
            fence_proxy_async();
            if (q == 0)
                bulk_s2g(grow + c * 16, s_addr, 128);
            else
                bulk_add_s2g_f64(grow + c * 16, s_addr, 128);
            bulk_commit();
        }
        tc_fence_before();
        arrive_empty(b);
    }
    bulk_wait_all();
}

// Ray stager role (one warp): stages the ray blocks rb0 .. rb0 + nrb - 1 in a
// ring of kFRayBufs shared-memory buffers.
__device__ __forceinline__ void stage_rays_role(const FusedArgs& g, int lane, int rb0, int nrb,
                                                unsigned char* rays_smem, uint64_t* ray_full,
                                                uint64_t* ray_empty, volatile int* flag) {
    using namespace sm100;
    // Ray stager: lane l stages ray l of each block as (z, x) pairs for
    // the packed phase: {zh, xh, zl, xl}, {zf, xf, es_re, es_im}
    // (coordinates relative to the screen centre, amplitude scaled). The
    // next block's loads are in flight while the stager waits for its
    // buffer to be released.
    for (int i = 0; i < nrb; ++i) {
        const int rb = i % kFRayBufs;
        const size_t j = (size_t)(rb0 + i) * kFRays + lane;
        double x = g.ox, z = g.oz, er = 0.0, ei = 0.0;
        if (j < g.n) {
            x = __ldg(g.rx + j);
            z = __ldg(g.rz + j);
            er = __ldg(g.er + j);
            ei = __ldg(g.ei + j);
        }
        if (i >= kFRayBufs &&
            !mbar_wait(&ray_empty[rb], (uint32_t)(i / kFRayBufs - 1) & 1u, g.wait_limit))
            *flag = 1;
        float xh, xl, xf, zh, zl, zf;
        split_coord(x - g.ox, g.a_turns, &xh, &xl, &xf);
        split_coord(z - g.oz, g.a_turns, &zh, &zl, &zf);
        float4* st = reinterpret_cast<float4*>(rays_smem + rb * kFRayBytes);
        st[2 * lane] = make_float4(zh, xh, zl, xl);
        st[2 * lane + 1] = make_float4(zf, xf, (float)(er * g.inv_scale), (float)(ei * g.inv_scale));
        __syncwarp();
        if (lane == 0) mbar_arrive(&ray_full[rb]);
    }
}

__global__ void __launch_bounds__(kFThreads, 1) fresnel_fused_kernel(FusedArgs g) {
    using namespace sm100;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* tiles = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(tiles + kFStages * kFStage);
    uint64_t* empty = full + kFStages;
    uint64_t* acc_full = empty + kFStages;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* ray_full = acc_empty + 2;
    uint64_t* ray_empty = ray_full + kFRayBufs;
    uint64_t* mma_done = ray_empty + kFRayBufs;  // every issued MMA has completed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    unsigned char* rays_smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(tmem_slot) + 64 + 15) & ~static_cast<uintptr_t>(15));

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x, nt = blockIdx.y, sp = blockIdx.z;
    const int rb0 = (int)((long long)g.ray_blocks * sp / g.splits);
    const int rb1 = (int)((long long)g.ray_blocks * (sp + 1) / g.splits);
    const int nrb = rb1 - rb0;
    const int nseg = (nrb + kFSeg - 1) / kFSeg;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kFStages; ++s) {
            mbar_init(&full[s], kFProdThreads / 32 + (s == 0 ? g.stall : 0u));  // per producer warp
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kFEpiThreads);
        }
        for (int b = 0; b < kFRayBufs; ++b) {
            mbar_init(&ray_full[b], 1);                      // the stager warp
            mbar_init(&ray_empty[b], kFProdThreads / 32);  // one arrival per producer warp
        }
        mbar_init(mma_done, 1);
        mbar_init_fence();
        *flag = 0;
    }
    if (warp == 0) tmem_alloc(tmem_slot, 2 * kFN);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // UMMA issuer: per ray block three K blocks (hi.hi, hi.lo, lo.hi);
            // segment q accumulates into buffer q & 1.
            constexpr uint32_t idesc = idesc_f16_f32(128, kFN);
            bool good = true;
            for (int q = 0; q < nseg && good; ++q) {
                const int b = q & 1, use = q >> 1;
                if (use >= 1 && !mbar_wait(&acc_empty[b], (uint32_t)(use - 1) & 1u, g.wait_limit)) {
                    *flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(b * kFN);
                const int i0 = q * kFSeg, i1 = min(nrb, i0 + kFSeg);
                for (int i = i0; i < i1; ++i) {
                    const int s = i % kFStages;
                    if (!mbar_wait(&full[s], (uint32_t)(i / kFStages) & 1u, g.wait_limit)) {
                        *flag = 1;
                        good = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_hi = smem_u32(tiles + (size_t)s * kFStage);
                    const uint32_t a_lo = a_hi + kFA, b_hi = a_hi + 2 * kFA, b_lo = b_hi + kFB;
                    const uint32_t as[3] = {a_hi, a_hi, a_lo}, bs[3] = {b_hi, b_lo, b_hi};
#pragma unroll
                    for (int p = 0; p < 3; ++p)
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            umma_f16(d, desc_kmajor_sw128(as[p] + 32u * k),
                                     desc_kmajor_sw128(bs[p] + 32u * k), idesc,
                                     (uint32_t)((i - i0) | p | k));
                    umma_commit(&empty[s]);
                }
                umma_commit(&acc_full[b]);
            }
            // A loop that gave up on a wait may leave MMAs in flight: wait
            // (bounded) for them before the accumulators are freed.
            umma_commit(mma_done);
            if (!mbar_wait(mma_done, 0, max(g.wait_limit, kMmaDrainPolls))) *flag = 1;
        }
        __syncwarp();
    } else if (warp <= 4) {
        unsigned char* tb = rays_smem + kFRayBufs * kFRayBytes + (warp - 1) * 32 * kFEpiRow;
        drain_role(g, warp, lane, mt, nt, sp, nseg, tmem, acc_full, tb, flag,
                   [&](int b) { mbar_arrive(&acc_empty[b]); });
    } else if (warp < 5 + kFProdThreads / 32) {
        // Producers: thread p owns kFRowsPer A rows r_k = (p % kFRowThreads) +
        // kFRowThreads k (screen z index mt*128 + r_k) and the B rows r_k,
        // 128 + r_k (screen x index nt*128 + r_k), for the 16-byte chunks
        // kFChunks q .. kFChunks (q + 1) - 1 (q = p / kFRowThreads) of each
        // ray block: every staged ray value a thread reads serves kFRowsPer
        // rows, and each store instruction of a warp covers 32 consecutive
        // rows. The stager warp stages each block's rays in shared memory up
        // to kFRayBufs blocks ahead.
        const int p = threadIdx.x - 160;
        const int q = p / kFRowThreads, rq = p % kFRowThreads;
        bool va[kFRowsPer], vb[kFRowsPer];
        // Per-row terms: kappa = -2 a p (hi, lo) and P = frac(a p^2), the A
        // row in .x and the B row in .y.
        float2 kh2[kFRowsPer], khn2[kFRowsPer], kl2[kFRowsPer], pp2[kFRowsPer];
#pragma unroll
        for (int k = 0; k < kFRowsPer; ++k) {
            const int r = rq + kFRowThreads * k;
            const size_t iz = (size_t)mt * 128 + r, ix = (size_t)nt * 128 + r;
            va[k] = iz < g.nz;
            vb[k] = ix < g.nx;
            const double zr = va[k] ? g.zp[iz] - g.oz : 0.0, xr = vb[k] ? g.xp[ix] - g.ox : 0.0;
            float kzh, kzl, kxh, kxl, pz, px, unused, h0, l0;
            split_coord(-2.0 * g.a_turns * zr, 0.0, &kzh, &kzl, &unused);
            split_coord(-2.0 * g.a_turns * xr, 0.0, &kxh, &kxl, &unused);
            split_coord(zr, g.a_turns, &h0, &l0, &pz);
            split_coord(xr, g.a_turns, &h0, &l0, &px);
            kh2[k] = make_float2(kzh, kxh);
            khn2[k] = make_float2(-kzh, -kxh);
            kl2[k] = make_float2(kzl, kxl);
            pp2[k] = make_float2(pz, px);
        }
        for (int i = 0; i < nrb; ++i) {
            const int s = i % kFStages, rb = i % kFRayBufs;
            bool ok = mbar_wait(&ray_full[rb], (uint32_t)(i / kFRayBufs) & 1u, g.wait_limit);
            ok = mbar_wait(&empty[s], ((uint32_t)(i / kFStages) & 1u) ^ 1u, g.wait_limit) && ok;
            if (!ok) *flag = 1;
            unsigned char* base = tiles + (size_t)s * kFStage;
            const float4* sr = reinterpret_cast<const float4*>(rays_smem + rb * kFRayBytes);
#pragma unroll 1
            for (int cc = 0; cc < kFChunks; ++cc) {
                const int c = kFChunks * q + cc;
                uint32_t ah[kFRowsPer][4], al[kFRowsPer][4], bh[kFRowsPer][4], bl[kFRowsPer][4];
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    const int j = 4 * c + jj;
                    const float4 v0 = sr[2 * j], v1 = sr[2 * j + 1];
#pragma unroll
                    for (int k = 0; k < kFRowsPer; ++k) {
                        // Phase in turns of the A row (.x) and the B row (.y).
                        const float2 t = pair_turns2(kh2[k], khn2[k], kl2[k],
                                                     __fadd2_rn(pp2[k], make_float2(v1.x, v1.y)),
                                                     make_float2(v0.x, v0.y),
                                                     make_float2(v0.z, v0.w));
                        const float2 th = __fmul2_rn(t, f2(6.28318530717958647692f));
                        float ca, sa, cb, sb, wr = 0.f, wi = 0.f;
                        __sincosf(th.x, &sa, &ca);
                        __sincosf(th.y, &sb, &cb);
                        if (!va[k]) ca = sa = 0.f;
                        if (vb[k]) {
                            wr = cmul_re(v1.z, v1.w, cb, sb);
                            wi = cmul_im(v1.z, v1.w, cb, sb);
                        }
                        split16x2(ca, sa, &ah[k][jj], &al[k][jj]);
                        split16x2(wr, wi, &bh[k][jj], &bl[k][jj]);
                    }
                }
                unsigned char* bhi = base + 2 * kFA;
                unsigned char* blo = bhi + kFB;
#pragma unroll
                for (int k = 0; k < kFRowsPer; ++k) {
                    const uint32_t r = (uint32_t)(rq + kFRowThreads * k);
                    // A row: (Re Z, Im Z); B rows r: (Re W, -Im W), 128 + r:
                    // (Im W, Re W). Each store instruction writes 32
                    // consecutive rows, which meet all eight swizzle phases
                    // (no bank conflict).
                    *reinterpret_cast<uint4*>(base + sw128(r, c)) =
                        make_uint4(ah[k][0], ah[k][1], ah[k][2], ah[k][3]);
                    *reinterpret_cast<uint4*>(base + kFA + sw128(r, c)) =
                        make_uint4(al[k][0], al[k][1], al[k][2], al[k][3]);
                    *reinterpret_cast<uint4*>(bhi + sw128(r, c)) =
                        make_uint4(neg_hi(bh[k][0]), neg_hi(bh[k][1]), neg_hi(bh[k][2]), neg_hi(bh[k][3]));
                    *reinterpret_cast<uint4*>(bhi + sw128(128 + r, c)) =
                        make_uint4(swap_halves(bh[k][0]), swap_halves(bh[k][1]),
                                   swap_halves(bh[k][2]), swap_halves(bh[k][3]));
                    *reinterpret_cast<uint4*>(blo + sw128(r, c)) =
                        make_uint4(neg_hi(bl[k][0]), neg_hi(bl[k][1]), neg_hi(bl[k][2]), neg_hi(bl[k][3]));
                    *reinterpret_cast<uint4*>(blo + sw128(128 + r, c)) =
                        make_uint4(swap_halves(bl[k][0]), swap_halves(bl[k][1]),
                                   swap_halves(bl[k][2]), swap_halves(bl[k][3]));
                }
            }
            // Make the generic-proxy stores visible to the tensor cores, then
            // one arrival per warp.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&full[s]);
                mbar_arrive(&ray_empty[rb]);
            }
        }
    } else {
        stage_rays_role(g, lane, rb0, nrb, rays_smem, ray_full, ray_empty, flag);
    }
    __syncthreads();
    if (*flag != 0 && threadIdx.x == 0) atomicExch(g.err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_free(tmem, 2 * kFN);
    }
}

// ---- the same product on CTA pairs (tcgen05 cta_group::2) ---------------------
//
// A cluster of two CTAs computes a 256 x 256 accumulator tile (256 z rows, 128
// x points) with one pair MMA per K step, issued by the even CTA: each CTA
// holds its 128 A rows and half of B (64 x points: their real parts in local
// rows 0..63, their imaginary parts in 64..127), and each keeps its 128
// accumulator rows in its own TMEM. Per 32-ray block a CTA therefore computes
// 128 A and 64 B phasors per ray instead of 128 + 128, stores 64 KB of tiles
// instead of 96 KB, and its tensor core reads half of B from each CTA. The
// accumulator column of x point ix is n = 128 h + 64 c + ix % 64 with
// h = (ix % 128) / 64 (the CTA that holds it) and c = 0 (real), 1 (imaginary).
constexpr int kPStages = 3;
constexpr uint32_t kPA = 128 * 128;              // one A tile (hi or lo): 128 rows x 128 B
constexpr uint32_t kPB = 128 * 128;              // this CTA's half of one B tile
constexpr uint32_t kPStage = 2 * kPA + 2 * kPB;  // A_hi | A_lo | B_hi | B_lo
constexpr int kPProdThreads = 384;               // warps 5..16
constexpr int kPThreads = 32 + kFEpiThreads + kPProdThreads + 32;
constexpr size_t kPSmem =
    1024 + (size_t)kPStages * kPStage + kFRayBufs * kFRayBytes + kFEpiBytes + 256;
static_assert(kPSmem <= 227 * 1024, "pair kernel shared memory");

// Producer warps of a CTA of the pair. Warps 0..7 (ZZ = false) fill 16-byte
// chunk c0 = w (rays 4 c0 .. 4 c0 + 3) of the A rows l, l + 32 and of the B
// rows of x points l, l + 32 (packed pair-rows (A l, B l), (A l+32, B l+32));
// warps 8..11 (ZZ = true) fill chunks c0, c0 + 1 of the A rows 64 + l, 96 + l
// (pair-row (A 64+l, A 96+l)). Every thread thus makes 8 packed phase
// evaluations per ray block; each store instruction of a warp covers 32
// consecutive rows (no bank conflict). Row z index mt*128 + row, x index
// nt*128 + 64 half + point.
template <bool ZZ>
__device__ __forceinline__ void pair_producer(const FusedArgs& g, int c0, int r, int mt, int nt,
                                              uint32_t half, int nrb, unsigned char* tiles,
                                              uint32_t full_lead, uint64_t* empty,
                                              uint64_t* ray_full, uint64_t* ray_empty,
                                              unsigned char* rays_smem, volatile int* flag) {
    using namespace sm100;
    constexpr int NE = ZZ ? 1 : 2;   // pair-rows per thread
    constexpr int NCH = ZZ ? 2 : 1;  // chunks per thread
    bool vx_ok[NE], vy_ok[NE];
    float2 kh2[NE], khn2[NE], kl2[NE], pp2[NE];
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        // (.x, .y) rows: (A r + 32 e, B r + 32 e) or (A 64 + r, A 96 + r).
        const size_t izx = (size_t)mt * 128 + (ZZ ? 64 + r : r + 32 * e);
        vx_ok[e] = izx < g.nz;
        const double ux = vx_ok[e] ? g.zp[izx] - g.oz : 0.0;
        double uy;
        if (ZZ) {
            const size_t izy = (size_t)mt * 128 + 96 + r;
            vy_ok[e] = izy < g.nz;
            uy = vy_ok[e] ? g.zp[izy] - g.oz : 0.0;
        } else {
            const size_t ix = (size_t)nt * 128 + 64 * half + r + 32 * e;
            vy_ok[e] = ix < g.nx;
            uy = vy_ok[e] ? g.xp[ix] - g.ox : 0.0;
        }
        float hx, lx, hy, ly, fx, fy, unused, h0, l0;
        split_coord(-2.0 * g.a_turns * ux, 0.0, &hx, &lx, &unused);
        split_coord(-2.0 * g.a_turns * uy, 0.0, &hy, &ly, &unused);
        split_coord(ux, g.a_turns, &h0, &l0, &fx);
        split_coord(uy, g.a_turns, &h0, &l0, &fy);
        kh2[e] = make_float2(hx, hy);
        khn2[e] = make_float2(-hx, -hy);
        kl2[e] = make_float2(lx, ly);
        pp2[e] = make_float2(fx, fy);
    }
    for (int i = 0; i < nrb; ++i) {
        const int s = i % kPStages, rb = i % kFRayBufs;
        bool ok = mbar_wait(&ray_full[rb], (uint32_t)(i / kFRayBufs) & 1u, g.wait_limit);
        ok = mbar_wait(&empty[s], ((uint32_t)(i / kPStages) & 1u) ^ 1u, g.wait_limit) && ok;
        if (!ok) *flag = 1;
        unsigned char* base = tiles + (size_t)s * kPStage;
        unsigned char* bhi = base + 2 * kPA;
        unsigned char* blo = bhi + kPB;
        const float4* sr = reinterpret_cast<const float4*>(rays_smem + rb * kFRayBytes);
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) {
            const int c = c0 + ch;
            // [row][ray]: A rows of .x and (ZZ) of .y; B points of .y.
            uint32_t ah[2][4], al[2][4], bh[2][4], bl[2][4];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                const int j = 4 * c + jj;
                const float4 v0 = sr[2 * j], v1 = sr[2 * j + 1];
                const float2 rh = ZZ ? f2(v0.x) : make_float2(v0.x, v0.y);
                const float2 rl = ZZ ? f2(v0.z) : make_float2(v0.z, v0.w);
                const float2 rf = ZZ ? f2(v1.x) : make_float2(v1.x, v1.y);
#pragma unroll
                for (int e = 0; e < NE; ++e) {
                    const float2 t = pair_turns2(kh2[e], khn2[e], kl2[e], __fadd2_rn(pp2[e], rf), rh, rl);
                    const float2 th = __fmul2_rn(t, f2(6.28318530717958647692f));
                    float sx, cx, sy, cy;
                    __sincosf(th.x, &sx, &cx);
                    __sincosf(th.y, &sy, &cy);
                    if (!vx_ok[e]) cx = sx = 0.f;
                    split16x2(cx, sx, &ah[ZZ ? 0 : e][jj], &al[ZZ ? 0 : e][jj]);
                    if (ZZ) {
                        if (!vy_ok[e]) cy = sy = 0.f;
                        split16x2(cy, sy, &ah[1][jj], &al[1][jj]);
                    } else {
                        float wr = 0.f, wi = 0.f;
                        if (vy_ok[e]) {
                            wr = cmul_re(v1.z, v1.w, cy, sy);
                            wi = cmul_im(v1.z, v1.w, cy, sy);
                        }
                        split16x2(wr, wi, &bh[e][jj], &bl[e][jj]);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const uint32_t row = (uint32_t)(ZZ ? 64 + r + 32 * k : r + 32 * k);
                *reinterpret_cast<uint4*>(base + sw128(row, c)) =
                    make_uint4(ah[k][0], ah[k][1], ah[k][2], ah[k][3]);
                *reinterpret_cast<uint4*>(base + kPA + sw128(row, c)) =
                    make_uint4(al[k][0], al[k][1], al[k][2], al[k][3]);
            }
            if (!ZZ) {
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    // Point r + 32 k: (Re W, -Im W) in row r + 32 k, (Im W,
                    // Re W) in row 64 + r + 32 k.
                    const uint32_t row = (uint32_t)(r + 32 * k);
                    *reinterpret_cast<uint4*>(bhi + sw128(row, c)) = make_uint4(
                        neg_hi(bh[k][0]), neg_hi(bh[k][1]), neg_hi(bh[k][2]), neg_hi(bh[k][3]));
                    *reinterpret_cast<uint4*>(bhi + sw128(64 + row, c)) =
                        make_uint4(swap_halves(bh[k][0]), swap_halves(bh[k][1]),
                                   swap_halves(bh[k][2]), swap_halves(bh[k][3]));
                    *reinterpret_cast<uint4*>(blo + sw128(row, c)) = make_uint4(
                        neg_hi(bl[k][0]), neg_hi(bl[k][1]), neg_hi(bl[k][2]), neg_hi(bl[k][3]));
                    *reinterpret_cast<uint4*>(blo + sw128(64 + row, c)) =
                        make_uint4(swap_halves(bl[k][0]), swap_halves(bl[k][1]),
                                   swap_halves(bl[k][2]), swap_halves(bl[k][3]));
                }
            }
        }
        // Make the generic-proxy stores visible to the tensor cores, then one
        // arrival per warp on the even CTA's stage barrier.
        fence_proxy_async();
        __syncwarp();
        if (r == 0) {
            mbar_arrive_cluster(full_lead + 8u * (uint32_t)s);
            mbar_arrive(&ray_empty[rb]);
        }
    }
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPThreads, 1)
    fresnel_pair_kernel(FusedArgs g) {
    using namespace sm100;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* tiles = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(tiles + kPStages * kPStage);
    uint64_t* empty = full + kPStages;
    uint64_t* acc_full = empty + kPStages;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* ray_full = acc_empty + 2;
    uint64_t* ray_empty = ray_full + kFRayBufs;
    uint64_t* mma_done = ray_empty + kFRayBufs;  // every issued MMA has completed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    unsigned char* rays_smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(tmem_slot) + 64 + 15) & ~static_cast<uintptr_t>(15));

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x, nt = blockIdx.y, sp = blockIdx.z;
    const uint32_t half = cluster_ctarank(), peer = half ^ 1u;
    const bool leader = half == 0;
    const int rb0 = (int)((long long)g.ray_blocks * sp / g.splits);
    const int rb1 = (int)((long long)g.ray_blocks * (sp + 1) / g.splits);
    const int nrb = rb1 - rb0;
    const int nseg = (nrb + kFSeg - 1) / kFSeg;

    if (threadIdx.x == 0) {
        // full and acc_empty are used in the even CTA only: they collect the
        // arrivals of both CTAs' producer and epilogue warps.
        for (int s = 0; s < kPStages; ++s) {
            mbar_init(&full[s], 2 * kPProdThreads / 32 + (s == 0 ? g.stall : 0u));
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 2 * kFEpiThreads);
        }
        for (int b = 0; b < kFRayBufs; ++b) {
            mbar_init(&ray_full[b], 1);
            mbar_init(&ray_empty[b], kPProdThreads / 32);
        }
        mbar_init(mma_done, 1);
        mbar_init_fence();
        *flag = 0;
    }
    if (warp == 0) tmem_alloc_pair(tmem_slot, 2 * kFN);
    tc_fence_before();
    cluster_sync();  // both CTAs' barriers initialised, TMEM allocated in both
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (leader && lane == 0) {
            // Pair MMA issuer: per ray block three K blocks (hi.hi, hi.lo,
            // lo.hi) of four 256x256x16 steps; segment q accumulates into
            // buffer q & 1 of both CTAs' TMEM.
            constexpr uint32_t idesc = idesc_f16_f32(256, kFN);
            bool good = true;
            for (int q = 0; q < nseg && good; ++q) {
                const int b = q & 1, use = q >> 1;
                if (use >= 1 &&
                    !mbar_wait_cluster(&acc_empty[b], (uint32_t)(use - 1) & 1u, g.wait_limit)) {
                    *flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(b * kFN);
                const int i0 = q * kFSeg, i1 = min(nrb, i0 + kFSeg);
                for (int i = i0; i < i1; ++i) {
                    const int s = i % kPStages;
                    if (!mbar_wait_cluster(&full[s], (uint32_t)(i / kPStages) & 1u, g.wait_limit)) {
                        *flag = 1;
                        good = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_hi = smem_u32(tiles + (size_t)s * kPStage);
                    const uint32_t a_lo = a_hi + kPA, b_hi = a_hi + 2 * kPA, b_lo = b_hi + kPB;
                    const uint32_t as[3] = {a_hi, a_hi, a_lo}, bs[3] = {b_hi, b_lo, b_hi};
#pragma unroll
                    for (int p = 0; p < 3; ++p)
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            umma_f16_pair(d, desc_kmajor_sw128(as[p] + 32u * k),
                                          desc_kmajor_sw128(bs[p] + 32u * k), idesc,
                                          (uint32_t)((i - i0) | p | k));
                    umma_commit_pair(smem_u32(&empty[s]));
                    umma_commit_pair(mapa_shared(&empty[s], peer));
                }
                umma_commit_pair(smem_u32(&acc_full[b]));
                umma_commit_pair(mapa_shared(&acc_full[b], peer));
            }
            // A loop that gave up on a wait may leave MMAs in flight: wait
            // (bounded) for them before either CTA frees its accumulators.
            umma_commit_pair(smem_u32(mma_done));
            if (!mbar_wait(mma_done, 0, max(g.wait_limit, kMmaDrainPolls))) *flag = 1;
        }
        __syncwarp();
    } else if (warp <= 4) {
        unsigned char* tb = rays_smem + kFRayBufs * kFRayBytes + (warp - 1) * 32 * kFEpiRow;
        const uint32_t acc_empty_lead = mapa_shared(acc_empty, 0);
        drain_role(g, warp, lane, mt, nt, sp, nseg, tmem, acc_full, tb, flag, [&](int b) {
            mbar_arrive_cluster(acc_empty_lead + 8u * (uint32_t)b);
        });
    } else if (warp < 5 + kPProdThreads / 32) {
        const int w = warp - 5;
        const uint32_t full_lead = mapa_shared(full, 0);
        if (w < 8)
            pair_producer<false>(g, w, lane, mt, nt, half, nrb, tiles, full_lead, empty, ray_full,
                                 ray_empty, rays_smem, flag);
        else
            pair_producer<true>(g, 2 * (w - 8), lane, mt, nt, half, nrb, tiles, full_lead, empty,
                                ray_full, ray_empty, rays_smem, flag);
    } else {
        stage_rays_role(g, lane, rb0, nrb, rays_smem, ray_full, ray_empty, flag);
    }
    __syncthreads();
    if (*flag != 0 && threadIdx.x == 0) atomicExch(g.err, 1);
    tc_fence_before();
    cluster_sync();  // the pair MMAs and all cross-CTA arrivals are done
    if (warp == 0) {
        tc_fence_after();
        tmem_free_pair(tmem, 2 * kFN);
    }
}

// acc[iz*nx + ix] (+)= scale * sum over splits of C[iz][n(ix, c)], in FP64 and
// split order.
// The ray set's bounds the product needs before it starts: max |es_re|,
// |es_im| (the f16 scaling), max |x - ox| and |z - oz| (the cross-term bound),
// and whether every value is finite. The maxima of non-negative doubles are
// taken on their bit patterns, which order like the values; fmax skips NaN,
// which the finiteness flag reports instead.
__global__ void __launch_bounds__(256) ray_bounds_kernel(const double* __restrict__ rx,
                                                         const double* __restrict__ rz,
                                                         const double* __restrict__ er,
                                                         const double* __restrict__ ei, size_t n,
                                                         double ox, double oz,
                                                         unsigned long long* __restrict__ max_bits,
                                                         int* __restrict__ nonfinite) {
    double m[3] = {0.0, 0.0, 0.0};
    bool bad = false;
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
         j += (size_t)gridDim.x * blockDim.x) {
        const double x = rx[j], z = rz[j], a = er[j], b = ei[j];
        m[0] = fmax(m[0], fmax(fabs(a), fabs(b)));
        m[1] = fmax(m[1], fabs(x - ox));
        m[2] = fmax(m[2], fabs(z - oz));
        bad = bad || !isfinite(x + z + a + b);
    }
    __shared__ double sm[8][3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double v = m[k];
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) sm[warp][k] = v;
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(nonfinite, 1);
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = sm[0][threadIdx.x];
        for (int w = 1; w < 8; ++w) v = fmax(v, sm[w][threadIdx.x]);
        atomicMax(max_bits + threadIdx.x, (unsigned long long)__double_as_longlong(v));
    }
}

// `group`: x points per real / imaginary column group of a 128-point block
// (128 for single-CTA tiles, 64 for CTA pairs).
__global__ void reduce_kernel(const double* __restrict__ partial, int splits, int m_pad, int n_pad,
                              int group, size_t nz, size_t nx, double scale,
                              double* __restrict__ acc_re, double* __restrict__ acc_im, int first) {
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (idx >= nz * nx) return;
    const size_t iz = idx / nx, ix = idx - iz * nx;
    const size_t loc = ix & 127, col = (ix >> 7) * kFN + 2 * group * (loc / group) + loc % group;
    double re = 0.0, im = 0.0;
    for (int s = 0; s < splits; ++s) {
        const double* row = partial + ((size_t)s * m_pad + iz) * n_pad + col;
        re += row[0];
        im += row[group];
    }
    re *= scale;
    im *= scale;
    if (first) {
        acc_re[idx] = re;
        acc_im[idx] = im;
    } else {
        acc_re[idx] += re;
        acc_im[idx] += im;
    }
}

// ---- host --------------------------------------------------------------------

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

unsigned grid_1d(size_t n, unsigned threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

FresnelShape fresnel_shape(size_t n, size_t nx, size_t nz, int num_sms, bool allow_pair) {
    FresnelShape sh;
    // CTA pairs need an even number of 128-row tiles; a screen of at most 128
    // rows keeps single-CTA tiles rather than padding to 256.
    sh.pair = allow_pair && nz > 128;
    sh.m_pad = round_up(std::max<size_t>(nz, 1), sh.pair ? 256 : 128);
    sh.n_pad = round_up(std::max<size_t>(2 * nx, 1), kFN);
    sh.ray_blocks = (int)((n + kFRays - 1) / kFRays);
    sh.tiles = (sh.m_pad / 128) * (sh.n_pad / kFN);
    // K splits: about one CTA per SM over the output tiles, each split at
    // least a few accumulation segments long.
    size_t splits = sh.tiles >= (size_t)num_sms ? 1 : (size_t)num_sms / sh.tiles;
    splits = std::min(splits, std::max<size_t>(1, (size_t)sh.ray_blocks / (2 * kFSeg)));
    sh.splits = (int)std::max<size_t>(1, splits);
    return sh;
}

Status fresnel_enqueue(const FresnelIn& in, FresnelWorkspace& ws, cudaStream_t stream,
                       int num_sms, int path, FresnelReport* rep) {
    const size_t n = in.n, nx = in.nx, nz = in.nz, m = nx * nz;
    double* xp = ws.coords.as<double>();
    double* zp = xp + std::max<size_t>(nx, 1);
    coords_kernel<<<grid_1d(nx, 256), 256, 0, stream>>>(in.x_min, in.x_max, nx, xp);
    coords_kernel<<<grid_1d(nz, 256), 256, 0, stream>>>(in.z_min, in.z_max, nz, zp);
    XK_CUDA_TRY(cudaGetLastError());
    rep->kernels += 2;
    const double k = in.energy / kChbar * 1e7;
    const double pre = k / (2.0 * in.dist);
    // Origin of the phase split and the bound on its FP32 cross term.
    const double ox = 0.5 * (in.x_min + in.x_max), oz = 0.5 * (in.z_min + in.z_max);
    const double cross = 2.0 * pre * kInv2Pi *
                         std::max(0.5 * std::fabs(in.x_max - in.x_min) * in.max_rx_off,
                                  0.5 * std::fabs(in.z_max - in.z_min) * in.max_rz_off);
    rep->used_path = path;
    // Non-finite inputs take the FP64 sum, which propagates them as
    // fresnel.rs:53-106 does.
    if (path == XK_PATH_SEPARABLE && n &&
        (!in.finite || (in.max_amp != 0.0 && !(cross < 2097152.0))))
        rep->used_path = path = XK_PATH_F64;
    if (path == XK_PATH_F64 || n == 0 || in.max_amp == 0.0) {
        // FP64 direct sum (with no rays or zero amplitudes it writes zeros).
        const size_t nn = (path == XK_PATH_F64) ? n : 0;
        fresnel_f64_kernel<<<grid_1d(m, kF64Threads), kF64Threads, 0, stream>>>(
            in.rx, in.rz, in.er, in.ei, nn, xp, zp, nx, m, pre, in.out_re, in.out_im);
        XK_CUDA_TRY(cudaGetLastError());
        rep->kernels += 1;
        return Status::Ok();
    }
    const FresnelShape sh = fresnel_shape(n, nx, nz, num_sms, ws.allow_pair);
    XK_TRY(ws.partial.ensure((size_t)sh.splits * sh.m_pad * sh.n_pad * sizeof(double)));
    XK_TRY(ws.ctrl.ensure(256));
    // Set on every call: the attribute belongs to the current device's
    // context, and a process may use several devices.
    if (sh.pair)
        XK_CUDA_TRY(cudaFuncSetAttribute(fresnel_pair_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPSmem));
    else
        XK_CUDA_TRY(cudaFuncSetAttribute(fresnel_fused_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFSmem));
    int* d_err = ws.ctrl.as<int>();
    XK_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    FusedArgs fa;
    fa.rx = in.rx;
    fa.rz = in.rz;
    fa.er = in.er;
    fa.ei = in.ei;
    fa.n = n;
    fa.ray_blocks = sh.ray_blocks;
    fa.splits = sh.splits;
    fa.xp = xp;
    fa.zp = zp;
    fa.nx = nx;
    fa.nz = nz;
    fa.a_turns = pre * kInv2Pi;
    fa.inv_scale = 1.0 / in.max_amp;
    fa.ox = ox;
    fa.oz = oz;
    fa.partial = ws.partial.as<double>();
    fa.m_pad = (int)sh.m_pad;
    fa.n_pad = (int)sh.n_pad;
    fa.err = d_err;
    fa.wait_limit = ws.wait_limit;
    fa.stall = ws.stall_once;
    ws.stall_once = 0;  // armed for one execution
    const dim3 grid((unsigned)(sh.m_pad / 128), (unsigned)(sh.n_pad / kFN), (unsigned)sh.splits);
    const bool timed = rep->ev_gemm[0] && rep->ev_gemm[1];
    if (timed) XK_CUDA_TRY(cudaEventRecord(rep->ev_gemm[0], stream));
    if (sh.pair)  // grid.x is even: m_pad is a multiple of 256
        fresnel_pair_kernel<<<grid, kPThreads, kPSmem, stream>>>(fa);
    else
        fresnel_fused_kernel<<<grid, kFThreads, kFSmem, stream>>>(fa);
    XK_CUDA_TRY(cudaGetLastError());
    if (timed) XK_CUDA_TRY(cudaEventRecord(rep->ev_gemm[1], stream));
    reduce_kernel<<<grid_1d(m, 256), 256, 0, stream>>>(ws.partial.as<double>(), sh.splits,
                                                        (int)sh.m_pad, (int)sh.n_pad,
                                                        sh.pair ? 64 : 128, nz, nx,
                                                        in.max_amp, in.out_re, in.out_im, 1);
    XK_CUDA_TRY(cudaGetLastError());
    rep->kernels += 2;
    if (timed) {
        XK_CUDA_TRY(cudaEventSynchronize(rep->ev_gemm[1]));
        float ms = 0.f;
        XK_CUDA_TRY(cudaEventElapsedTime(&ms, rep->ev_gemm[0], rep->ev_gemm[1]));
        rep->gemm_ms += ms;
    }
    rep->shape = sh;
    rep->d_err = d_err;
    return Status::Ok();
}

}  // namespace xk

// ---- C ABI -------------------------------------------------------------------

namespace {

int fr_fail(xk_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

xk::Status fresnel_host(xk_ctx* ctx, const double* rx, const double* rz, const double* er,
                        const double* ei, size_t n, double energy, double dist,
                        const xk_fresnel_screen* sc, double* amp_re, double* amp_im,
                        double* x_pixels, double* z_pixels, int path, xk_stats* stats) {
    cudaStream_t s = ctx->stream;
    xk::FresnelWorkspace& ws = ctx->fresnel;
    const size_t nx = sc->nx, nz = sc->nz, m = nx * nz;
    const size_t nb = n * sizeof(double);
    XK_TRY(ctx->in_rays.ensure(std::max<size_t>(4 * nb, 8)));
    XK_TRY(ws.coords.ensure((std::max<size_t>(nx, 1) + std::max<size_t>(nz, 1)) * sizeof(double)));
    XK_TRY(ctx->out_field.ensure(std::max<size_t>(2 * m * sizeof(double), 8)));
    double* d = ctx->in_rays.as<double>();
    const double* src[4] = {rx, rz, er, ei};
    for (int f = 0; f < 4 && n; ++f)
        XK_CUDA_TRY(cudaMemcpyAsync(d + f * n, src[f], nb, cudaMemcpyHostToDevice, s));
    double max_amp = 0.0, max_rx = 0.0, max_rz = 0.0;
    const double ox = 0.5 * (sc->x_min + sc->x_max), oz = 0.5 * (sc->z_min + sc->z_max);
    bool finite = true;
    int bounds_kernels = 0;
    if (n) {
        // The bounds come from the uploaded columns on the device (a host
        // loop over 2^20 rays takes milliseconds); one small read-back.
        XK_TRY(ws.ctrl.ensure(256));
        unsigned long long* d_max = reinterpret_cast<unsigned long long*>(ws.ctrl.as<char>() + 64);
        int* d_bad = reinterpret_cast<int*>(d_max + 3);
        XK_CUDA_TRY(cudaMemsetAsync(d_max, 0, 3 * sizeof(unsigned long long) + sizeof(int), s));
        const unsigned blocks =
            (unsigned)std::min<size_t>((n + 255) / 256, (size_t)std::max(ctx->num_sms, 1) * 4);
        xk::ray_bounds_kernel<<<blocks, 256, 0, s>>>(d, d + n, d + 2 * n, d + 3 * n, n, ox, oz,
                                                     d_max, d_bad);
        XK_CUDA_TRY(cudaGetLastError());
        bounds_kernels = 1;
        struct {
            unsigned long long m[3];
            int bad;
        } h{};
        XK_CUDA_TRY(cudaMemcpyAsync(&h, d_max, sizeof(h.m) + sizeof(int),
                                    cudaMemcpyDeviceToHost, s));
        XK_CUDA_TRY(cudaStreamSynchronize(s));
        double v[3];
        std::memcpy(v, h.m, sizeof(v));
        // An upper bound of |es_j| is all the f16 scaling needs.
        max_amp = v[0];
        max_rx = v[1];
        max_rz = v[2];
        finite = h.bad == 0;
    }
    max_amp *= 1.4142135623730951;
    double* out = ctx->out_field.as<double>();
    xk::FresnelIn in{d, d + n, d + 2 * n, d + 3 * n, n, energy, dist,
                     sc->x_min, sc->x_max, sc->z_min, sc->z_max, nx, nz, max_amp, max_rx, max_rz,
                     out, out + m, finite};
    xk::FresnelReport rep;
    cudaEvent_t g0 = nullptr, g1 = nullptr;
    if (stats && path == XK_PATH_SEPARABLE) {
        XK_CUDA_TRY(cudaEventCreate(&g0));
        XK_CUDA_TRY(cudaEventCreate(&g1));
        rep.ev_gemm[0] = g0;
        rep.ev_gemm[1] = g1;
    }
    XK_CUDA_TRY(cudaEventRecord(ctx->ev0, s));
    xk::Status st = xk::fresnel_enqueue(in, ws, s, ctx->num_sms, path, &rep);
    if (st.ok()) st = xk::Status::FromCuda(cudaEventRecord(ctx->ev1, s));
    int h_err = 0;
    if (st.ok() && rep.d_err)
        st = xk::Status::FromCuda(cudaMemcpyAsync(&h_err, rep.d_err, sizeof(int),
                                                  cudaMemcpyDeviceToHost, s));
    if (st.ok()) {
        st = xk::Status::FromCuda(cudaMemcpyAsync(amp_re, out, m * sizeof(double),
                                                  cudaMemcpyDeviceToHost, s));
        if (st.ok())
            st = xk::Status::FromCuda(cudaMemcpyAsync(amp_im, out + m, m * sizeof(double),
                                                      cudaMemcpyDeviceToHost, s));
        const double* xp = ws.coords.as<double>();
        if (st.ok() && x_pixels && nx)
            st = xk::Status::FromCuda(cudaMemcpyAsync(x_pixels, xp, nx * sizeof(double),
                                                      cudaMemcpyDeviceToHost, s));
        if (st.ok() && z_pixels && nz)
            st = xk::Status::FromCuda(cudaMemcpyAsync(z_pixels, xp + std::max<size_t>(nx, 1),
                                                      nz * sizeof(double),
                                                      cudaMemcpyDeviceToHost, s));
    }
    if (st.ok()) st = xk::Status::FromCuda(cudaStreamSynchronize(s));
    if (g0) cudaEventDestroy(g0);
    if (g1) cudaEventDestroy(g1);
    XK_TRY(st);
    if (h_err) return xk::Status::Err(XK_ERR_TIMEOUT, "tensor-core product: a bounded wait ran out");
    if (stats) {
        float ms = 0.f;
        XK_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        stats->gpu_ms = ms;
        stats->main_kernel_ms = rep.gemm_ms;
        stats->kernels = rep.kernels + bounds_kernels;
        stats->path = rep.used_path;
        stats->pairs = (double)n * (double)m;
        stats->h2d_bytes = 4.0 * nb;
        stats->d2h_bytes = 2.0 * m * sizeof(double) + (double)(nx + nz) * sizeof(double);
        stats->n_chunks = rep.shape.ray_blocks;
        stats->n_tiles = (int)rep.shape.tiles;
        stats->groups = rep.shape.splits;
        stats->n_items = (long long)rep.shape.tiles * rep.shape.splits;
        stats->sweep = rep.used_path == XK_PATH_SEPARABLE ? (rep.shape.pair ? 1 : 0) : -1;
    }
    return xk::Status::Ok();
}

}  // namespace

extern "C" int xk_fresnel_propagate(xk_ctx* ctx, const double* ray_x, const double* ray_z,
                                    const double* es_re, const double* es_im, size_t n_rays,
                                    double energy, double dist, const xk_fresnel_screen* screen,
                                    double* amp_re, double* amp_im, double* x_pixels,
                                    double* z_pixels, int path, xk_stats* stats) {
    if (!ctx) return XK_ERR_INVALID;
    if (!screen) return fr_fail(ctx, XK_ERR_INVALID, "null screen");
    if (path != XK_PATH_F64 && path != XK_PATH_SEPARABLE)
        return fr_fail(ctx, XK_ERR_INVALID, "unknown path (F64 or SEPARABLE)");
    const size_t nx = screen->nx, nz = screen->nz;
    if (nx && nz > SIZE_MAX / nx) return fr_fail(ctx, XK_ERR_INVALID, "nx * nz overflows");
    if (nx > (size_t)1 << 30 || nz > (size_t)1 << 30)
        return fr_fail(ctx, XK_ERR_INVALID, "screen too large");
    auto t0 = std::chrono::steady_clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (nx * nz == 0) return XK_OK;
    if (n_rays && (!ray_x || !ray_z || !es_re || !es_im))
        return fr_fail(ctx, XK_ERR_INVALID, "null ray array");
    if (!amp_re || !amp_im) return fr_fail(ctx, XK_ERR_INVALID, "null output array");
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    xk::Status st = fresnel_host(ctx, ray_x, ray_z, es_re, es_im, n_rays, energy, dist, screen,
                                 amp_re, amp_im, x_pixels, z_pixels, path, stats);
    if (!st.ok()) return fr_fail(ctx, st.code, st.msg);
    if (stats)
        stats->wall_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                .count();
    return XK_OK;
}
