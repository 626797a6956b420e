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
//       C[iz][2 ix + c] = sum_k A[iz][k] B[2 ix + c][k],
//       A[iz][2j] = Re Z, A[iz][2j+1] = Im Z,
//       B[2ix][2j] = Re W, B[2ix][2j+1] = -Im W, B[2ix+1][2j] = Im W, B[2ix+1][2j+1] = Re W,
//   with W = es X / max|es|. The factors (unit phasors, phases in FP64) are
//   written in f16 as hi + lo pairs and multiplied on the tensor cores
//   (tcgen05.mma kind::f16, f32 accumulators in tensor memory) as
//   A_hi B_hi + A_hi B_lo + A_lo B_hi (three K-blocks of one product), which
//   keeps ~2^-22 of each phasor; rays are processed in chunks, each chunk's
//   K range split across CTAs, and split and chunk partials are added in
//   FP64 in a fixed order (results do not depend on scheduling).
//
// The GEMM kernel: one CTA per 128 x 256 output tile and K range, 192
// threads; thread 0 issues TMA loads of 128x64 (A) and 256x64 (B) f16 tiles
// with the 128-byte swizzle into a 4-stage ring, thread 32 issues four
// 128x256x16 UMMAs per stage and commits each stage back to the producer;
// every kSeg stages the accumulator (one of two in tensor memory) is handed
// to four epilogue warps, which read it out (one 32-lane quarter each) and
// add it into the CTA's FP64 split partial while the next segment runs.

#include <cuda.h>
#include <cudaTypedefs.h>
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

// ---- separable product on the tensor cores -----------------------------------

constexpr int kBM = 128, kBN = 256, kBK = 64, kStages = 4;
constexpr uint32_t kABytes = kBM * kBK * 2, kBBytes = kBN * kBK * 2;
constexpr uint32_t kStageBytes = kABytes + kBBytes;
constexpr size_t kGemmSmem = 1024 + (size_t)kStages * kStageBytes + 256;
constexpr int kEpiThreads = 128;                 // four epilogue warps
constexpr int kGemmThreads = 64 + kEpiThreads;   // producer warp, UMMA warp, epilogue
constexpr int kSeg = 32;                         // K blocks per f32 accumulation segment

// exp(i a (p - r)^2) with the phase formed in FP64 and reduced to turns.
__device__ __forceinline__ void phasor(double p, double r, double a, double* c, double* s) {
    const double d = p - r;
    const double turns = a * d * d * kInv2Pi;
    const double f = turns - rint(turns);
    sincospi(2.0 * f, s, c);
}

__device__ __forceinline__ void split_h(double v, __half* hi, __half* lo) {
    *hi = __double2half(v);
    *lo = __double2half(v - (double)__half2float(*hi));
}

// A rows (screen z): row iz of K3 = 6 kc halves, ray j of the chunk at
// columns 2j (re), 2j+1 (im) of each of the three K blocks [hi | hi | lo].
__global__ void factor_a_kernel(const double* __restrict__ zp, size_t nz,
                                const double* __restrict__ rz, size_t n, size_t j0, size_t kc,
                                double a, __half* __restrict__ A, size_t K3) {
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (idx >= nz * kc) return;
    const size_t iz = idx / kc, j = idx - iz * kc, jj = j0 + j;
    double c = 0.0, s = 0.0;
    if (jj < n) phasor(zp[iz], rz[jj], a, &c, &s);
    __half ch, cl, sh, sl;
    split_h(c, &ch, &cl);
    split_h(s, &sh, &sl);
    __half2* row = reinterpret_cast<__half2*>(A + iz * K3);
    row[j] = __halves2half2(ch, sh);
    row[kc + j] = __halves2half2(ch, sh);
    row[2 * kc + j] = __halves2half2(cl, sl);
}

// B rows (screen x, two per point): [hi | lo | hi] blocks of the W matrix.
__global__ void factor_b_kernel(const double* __restrict__ xp, size_t nx,
                                const double* __restrict__ rx, const double* __restrict__ er,
                                const double* __restrict__ ei, size_t n, size_t j0, size_t kc,
                                double a, double inv_scale, __half* __restrict__ B, size_t K3) {
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (idx >= nx * kc) return;
    const size_t ix = idx / kc, j = idx - ix * kc, jj = j0 + j;
    double wr = 0.0, wi = 0.0;
    if (jj < n) {
        double c, s;
        phasor(xp[ix], rx[jj], a, &c, &s);
        const double e_r = er[jj] * inv_scale, e_i = ei[jj] * inv_scale;
        wr = e_r * c - e_i * s;
        wi = e_r * s + e_i * c;
    }
    __half rh, rl, ih, il, nih, nil;
    split_h(wr, &rh, &rl);
    split_h(wi, &ih, &il);
    nih = __hneg(ih);
    nil = __hneg(il);
    __half2* r0 = reinterpret_cast<__half2*>(B + (2 * ix) * K3);
    __half2* r1 = reinterpret_cast<__half2*>(B + (2 * ix + 1) * K3);
    r0[j] = __halves2half2(rh, nih);
    r0[kc + j] = __halves2half2(rl, nil);
    r0[2 * kc + j] = __halves2half2(rh, nih);
    r1[j] = __halves2half2(ih, rh);
    r1[kc + j] = __halves2half2(il, rl);
    r1[2 * kc + j] = __halves2half2(ih, rh);
}

// partial[split][m][n] (FP64) = A[m, K range] * B[n, K range]^T.
//
// The tensor cores accumulate in f32; over long K ranges their accumulation
// error grows with the number of accumulated blocks, so the K range is
// processed in segments of kSeg blocks, each into a fresh accumulator, and
// every finished segment is drained into the FP64 partial. Two accumulators
// (512 TMEM columns) alternate: the UMMA thread fills one while the four
// epilogue warps drain the other.
__global__ void __launch_bounds__(kGemmThreads, 1)
fresnel_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    int kb_total, int splits, double* __restrict__ partial, int m_pad, int n_pad,
                    int* __restrict__ err) {
    using namespace sm100;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* tiles = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(tiles + kStages * kStageBytes);
    uint64_t* empty = full + kStages;
    uint64_t* acc_full = empty + kStages;
    uint64_t* acc_empty = acc_full + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
    volatile int* flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x, nt = blockIdx.y, sp = blockIdx.z;
    const int kb0 = (int)((long long)kb_total * sp / splits);
    const int kb1 = (int)((long long)kb_total * (sp + 1) / splits);
    const int nkb = kb1 - kb0;
    const int nseg = (nkb + kSeg - 1) / kSeg;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kEpiThreads);
        }
        mbar_init_fence();
        *flag = 0;
        prefetch_tensor_map(&tmA);
        prefetch_tensor_map(&tmB);
    }
    if (warp == 1) tmem_alloc(tmem_slot, 2 * kBN);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0) {
        // TMA producer over the whole K range.
        for (int i = 0; i < nkb; ++i) {
            const int s = i % kStages;
            const uint32_t ph = (uint32_t)(i / kStages) & 1u;
            if (!mbar_wait(&empty[s], ph ^ 1u)) {
                *flag = 1;
                break;
            }
            mbar_arrive_expect_tx(&full[s], kStageBytes);
            unsigned char* a = tiles + (size_t)s * kStageBytes;
            const int kx = (kb0 + i) * kBK;
            tma_load_2d(a, &tmA, kx, mt * kBM, &full[s]);
            tma_load_2d(a + kABytes, &tmB, kx, nt * kBN, &full[s]);
        }
    } else if (threadIdx.x == 32) {
        // UMMA issuer: segment g accumulates into buffer g & 1.
        constexpr uint32_t idesc = idesc_f16_f32(kBM, kBN);
        bool good = true;
        for (int g = 0; g < nseg && good; ++g) {
            const int b = g & 1, use = g >> 1;
            if (use >= 1 && !mbar_wait(&acc_empty[b], (uint32_t)(use - 1) & 1u)) {
                *flag = 1;
                break;
            }
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(b * kBN);
            const int i0 = g * kSeg, i1 = min(nkb, i0 + kSeg);
            for (int i = i0; i < i1; ++i) {
                const int s = i % kStages;
                const uint32_t ph = (uint32_t)(i / kStages) & 1u;
                if (!mbar_wait(&full[s], ph)) {
                    *flag = 1;
                    good = false;
                    break;
                }
                tc_fence_after();
                const uint32_t a = smem_u32(tiles + (size_t)s * kStageBytes);
                const uint32_t bb = a + kABytes;
#pragma unroll
                for (int k = 0; k < kBK / 16; ++k)
                    umma_f16(d, desc_kmajor_sw128(a + 32u * k), desc_kmajor_sw128(bb + 32u * k),
                             idesc, (uint32_t)((i - i0) | k));
                umma_commit(&empty[s]);
            }
            umma_commit(&acc_full[b]);  // arrives once the segment's UMMAs have completed
        }
    } else if (warp >= 2) {
        // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its quarter).
        const int q = warp & 3;
        const int row = mt * kBM + q * 32 + lane;
        double* dst = partial + ((size_t)sp * m_pad + row) * n_pad + (size_t)nt * kBN;
        if (nseg == 0) {
            for (int c = 0; c < kBN; c += 2)
                *reinterpret_cast<double2*>(dst + c) = make_double2(0.0, 0.0);
        }
        for (int g = 0; g < nseg; ++g) {
            const int b = g & 1;
            const bool ok = mbar_wait(&acc_full[b], (uint32_t)(g >> 1) & 1u);
            if (!__all_sync(0xffffffffu, ok)) {
                *flag = 1;
                break;
            }
            tc_fence_after();
#pragma unroll 1
            for (int c = 0; c < kBN / 32; ++c) {
                float v[32];
                tmem_ld_32cols(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kBN + c * 32), v);
                double2* d2 = reinterpret_cast<double2*>(dst + c * 32);
                if (g == 0) {
#pragma unroll
                    for (int t = 0; t < 16; ++t)
                        d2[t] = make_double2((double)v[2 * t], (double)v[2 * t + 1]);
                } else {
#pragma unroll
                    for (int t = 0; t < 16; ++t) {
                        double2 o = d2[t];
                        o.x += (double)v[2 * t];
                        o.y += (double)v[2 * t + 1];
                        d2[t] = o;
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&acc_empty[b]);
        }
    }
    __syncthreads();
    if (*flag != 0 && threadIdx.x == 0) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_free(tmem, 2 * kBN);
    }
}

// acc[iz*nx + ix] (+)= scale * sum over splits of C[iz][2ix + c], in FP64 and
// split order.
__global__ void reduce_kernel(const double* __restrict__ partial, int splits, int m_pad, int n_pad,
                              size_t nz, size_t nx, double scale, double* __restrict__ acc_re,
                              double* __restrict__ acc_im, int first) {
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (idx >= nz * nx) return;
    const size_t iz = idx / nx, ix = idx - iz * nx;
    double re = 0.0, im = 0.0;
    for (int s = 0; s < splits; ++s) {
        const double2 v = *reinterpret_cast<const double2*>(
            partial + ((size_t)s * m_pad + iz) * n_pad + 2 * ix);
        re += v.x;
        im += v.y;
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

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Row-major [rows][k] f16 matrix, tiles of box_rows x 64 with the 128-byte swizzle.
Status make_map(CUtensorMap* map, const void* base, size_t k, size_t rows, uint32_t box_rows) {
    auto fn = encode_fn();
    if (!fn) return Status::Err(XK_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(k * 2)};
    cuuint32_t box[2] = {(cuuint32_t)kBK, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return Status::Err(XK_ERR_CUDA, "tensor map encoding failed");
    return Status::Ok();
}

}  // namespace

FresnelShape fresnel_shape(size_t n, size_t nx, size_t nz, int num_sms, size_t factor_budget,
                           size_t max_chunk_rays) {
    FresnelShape sh;
    sh.m_pad = round_up(std::max<size_t>(nz, 1), kBM);
    sh.n_pad = round_up(std::max<size_t>(2 * nx, 1), kBN);
    // Rays per chunk: a multiple of 32 (K3 = 6 kc is then a multiple of the
    // 64-wide K block) within the factor-memory budget.
    const size_t per_ray = 12 * (sh.m_pad + sh.n_pad);  // bytes of A and B per ray
    size_t kc = std::max<size_t>(32, factor_budget / per_ray / 32 * 32);
    if (max_chunk_rays) kc = std::min(kc, std::max<size_t>(32, max_chunk_rays / 32 * 32));
    kc = std::min(kc, round_up(std::max<size_t>(n, 1), 32));
    sh.kc = kc;
    sh.chunks = (n + kc - 1) / kc;
    sh.k3 = 6 * kc;
    sh.kb_total = (int)(sh.k3 / kBK);
    const size_t tiles = (sh.m_pad / kBM) * (sh.n_pad / kBN);
    size_t splits = tiles >= (size_t)num_sms ? 1 : (size_t)num_sms / tiles;
    splits = std::max<size_t>(1, std::min(splits, (size_t)std::max(1, sh.kb_total / 4)));
    sh.splits = (int)splits;
    sh.tiles = tiles;
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
    if (path == XK_PATH_F64 || n == 0 || in.max_amp == 0.0) {
        // FP64 direct sum (with no rays or zero amplitudes it writes zeros).
        const size_t nn = (path == XK_PATH_F64) ? n : 0;
        fresnel_f64_kernel<<<grid_1d(m, kF64Threads), kF64Threads, 0, stream>>>(
            in.rx, in.rz, in.er, in.ei, nn, xp, zp, nx, m, pre, in.out_re, in.out_im);
        XK_CUDA_TRY(cudaGetLastError());
        rep->kernels += 1;
        return Status::Ok();
    }
    const FresnelShape sh = fresnel_shape(n, nx, nz, num_sms, ws.factor_budget, ws.max_chunk_rays);
    XK_TRY(ws.factors.ensure((sh.m_pad + sh.n_pad) * sh.k3 * sizeof(__half)));
    XK_TRY(ws.partial.ensure((size_t)sh.splits * sh.m_pad * sh.n_pad * sizeof(double)));
    XK_TRY(ws.ctrl.ensure(256));
    __half* A = ws.factors.as<__half>();
    __half* B = A + sh.m_pad * sh.k3;
    CUtensorMap mapA, mapB;
    XK_TRY(make_map(&mapA, A, sh.k3, sh.m_pad, kBM));
    XK_TRY(make_map(&mapB, B, sh.k3, sh.n_pad, kBN));
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
        attr_err = cudaFuncSetAttribute(fresnel_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kGemmSmem);
    });
    XK_CUDA_TRY(attr_err);
    int* d_err = ws.ctrl.as<int>();
    XK_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    // Padding rows of A and B stay zero for every chunk.
    XK_CUDA_TRY(cudaMemsetAsync(ws.factors.ptr, 0, (sh.m_pad + sh.n_pad) * sh.k3 * sizeof(__half),
                                stream));
    const double inv_scale = 1.0 / in.max_amp;
    const dim3 grid((unsigned)(sh.m_pad / kBM), (unsigned)(sh.n_pad / kBN), (unsigned)sh.splits);
    for (size_t c = 0; c < sh.chunks; ++c) {
        const size_t j0 = c * sh.kc;
        factor_a_kernel<<<grid_1d(nz * sh.kc, 256), 256, 0, stream>>>(zp, nz, in.rz, n, j0, sh.kc,
                                                                       pre, A, sh.k3);
        factor_b_kernel<<<grid_1d(nx * sh.kc, 256), 256, 0, stream>>>(
            xp, nx, in.rx, in.er, in.ei, n, j0, sh.kc, pre, inv_scale, B, sh.k3);
        XK_CUDA_TRY(cudaGetLastError());
        const bool timed = rep->ev_gemm[0] && rep->ev_gemm[1];
        if (timed) XK_CUDA_TRY(cudaEventRecord(rep->ev_gemm[0], stream));
        fresnel_gemm_kernel<<<grid, kGemmThreads, kGemmSmem, stream>>>(
            mapA, mapB, sh.kb_total, sh.splits, ws.partial.as<double>(), (int)sh.m_pad,
            (int)sh.n_pad, d_err);
        XK_CUDA_TRY(cudaGetLastError());
        if (timed) {
            XK_CUDA_TRY(cudaEventRecord(rep->ev_gemm[1], stream));
            XK_CUDA_TRY(cudaEventSynchronize(rep->ev_gemm[1]));
            float ms = 0.f;
            XK_CUDA_TRY(cudaEventElapsedTime(&ms, rep->ev_gemm[0], rep->ev_gemm[1]));
            rep->gemm_ms += ms;
        }
        reduce_kernel<<<grid_1d(m, 256), 256, 0, stream>>>(ws.partial.as<double>(), sh.splits,
                                                            (int)sh.m_pad, (int)sh.n_pad, nz, nx,
                                                            in.max_amp, in.out_re, in.out_im,
                                                            c == 0);
        XK_CUDA_TRY(cudaGetLastError());
        rep->kernels += 4;
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
    double max_amp = 0.0;
    for (size_t j = 0; j < n; ++j) max_amp = std::max(max_amp, std::hypot(er[j], ei[j]));
    double* out = ctx->out_field.as<double>();
    xk::FresnelIn in{d, d + n, d + 2 * n, d + 3 * n, n, energy, dist,
                     sc->x_min, sc->x_max, sc->z_min, sc->z_max, nx, nz, max_amp, out, out + m};
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
        stats->kernels = rep.kernels;
        stats->path = path;
        stats->pairs = (double)n * (double)m;
        stats->h2d_bytes = 4.0 * nb;
        stats->d2h_bytes = 2.0 * m * sizeof(double) + (double)(nx + nz) * sizeof(double);
        stats->n_chunks = (int)rep.shape.chunks;
        stats->n_tiles = (int)rep.shape.tiles;
        stats->groups = rep.shape.splits;
        stats->n_items = (long long)rep.shape.tiles * rep.shape.splits * (long long)rep.shape.chunks;
        stats->sweep = -1;
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
