// Pipe throughput probe: the FP32 FMA pipe and the MUFU (SFU) unit.
//
// The phase-reduced pair kernel is bound by these two pipes, not by HBM or
// the tensor cores, so its roofline needs their peak rates on this part.
// Two kernels measure them with every SM busy:
//   * ffma2_probe: 8 independent f32x2 FMA chains per thread, 32 warps per
//     SM (an f32x2 FMA counts as two lane operations);
//   * mufu_probe: 8 independent chains of sin.approx / cos.approx per thread
//     (each MUFU result counts once; the range multiply before each one runs
//     on the FMA pipe, far below its rate).
// One block of 1024 threads per SM (its shared-memory request keeps a second
// block off the SM), so a block's clock64 cycle count between entry and exit
// is its SM's: the rates come out per SM clock, independent of the clock the
// GPU happened to run at. CUDA events give the wall time, and cycles over
// time the SM clock seen.

#include <algorithm>
#include <vector>

#include "xk_ctx.cuh"

namespace xk {
namespace {

constexpr int kProbeThreads = 1024;
constexpr int kProbeBlocksPerSm = 1;
constexpr int kProbeChains = 8;
// Dynamic shared memory per block: more than half the SM's 228 KB, so every
// SM holds exactly one block of the num_sms-block grid.
constexpr int kProbeSmem = 120 * 1024;

__global__ void __launch_bounds__(kProbeThreads)
ffma2_probe(int iters, float seed, float* __restrict__ sink, long long* __restrict__ cycles) {
    float2 acc[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c)
        acc[c] = make_float2(seed + 0.001f * (float)(threadIdx.x + c), seed - 0.002f * (float)c);
    const float2 mul = make_float2(0.999999f, 1.000001f);
    const float2 add = make_float2(1e-7f, -1e-7f);
    __syncthreads();
    const long long t0 = clock64();
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int c = 0; c < kProbeChains; ++c) acc[c] = __ffma2_rn(acc[c], mul, add);
    }
    __syncthreads();
    const long long t1 = clock64();
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) s += acc[c].x + acc[c].y;
    if (s == 12345.678f) sink[threadIdx.x] = s;  // keeps the chains alive
    if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
}

__device__ __forceinline__ float sin_approx(float x) {
    float r;
    asm volatile("sin.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float cos_approx(float x) {
    float r;
    asm volatile("cos.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__global__ void __launch_bounds__(kProbeThreads)
mufu_probe(int iters, float seed, float* __restrict__ sink, long long* __restrict__ cycles) {
    float v[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) v[c] = seed + 0.01f * (float)(threadIdx.x & 31) + 0.1f * c;
    __syncthreads();
    const long long t0 = clock64();
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c) v[c] = sin_approx(v[c]);
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c) v[c] = cos_approx(v[c]);
    }
    __syncthreads();
    const long long t1 = clock64();
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) s += v[c];
    if (s == 12345.678f) sink[threadIdx.x] = s;
    if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
}

struct ProbeRun {
    double ops_per_clk_sm = 0.0;
    double ms = 0.0;
    double clk_mhz = 0.0;
};

// Runs `kern` on num_sms blocks (one per SM); ops_per_block lane operations
// per block; the rate uses the median block's cycle count.
template <class K>
Status run_probe(K kern, int iters, double ops_per_block, int num_sms, cudaStream_t s,
                 DevBuf& scratch, ProbeRun* out) {
    const int blocks = num_sms * kProbeBlocksPerSm;
    XK_TRY(scratch.ensure(blocks * sizeof(long long) + kProbeThreads * sizeof(float)));
    long long* d_cycles = scratch.as<long long>();
    float* d_sink = reinterpret_cast<float*>(d_cycles + blocks);
    cudaEvent_t e0, e1;
    XK_CUDA_TRY(cudaEventCreate(&e0));
    XK_CUDA_TRY(cudaEventCreate(&e1));
    XK_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kProbeSmem));
    kern<<<blocks, kProbeThreads, kProbeSmem, s>>>(iters / 8, 1.0f, d_sink, d_cycles);  // warm-up
    XK_CUDA_TRY(cudaGetLastError());
    XK_CUDA_TRY(cudaEventRecord(e0, s));
    kern<<<blocks, kProbeThreads, kProbeSmem, s>>>(iters, 1.0f, d_sink, d_cycles);
    XK_CUDA_TRY(cudaGetLastError());
    XK_CUDA_TRY(cudaEventRecord(e1, s));
    XK_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    XK_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::vector<long long> cyc(blocks);
    XK_CUDA_TRY(cudaMemcpy(cyc.data(), d_cycles, blocks * sizeof(long long), cudaMemcpyDeviceToHost));
    std::sort(cyc.begin(), cyc.end());
    const double med = (double)cyc[blocks / 2];
    out->ops_per_clk_sm = ops_per_block * kProbeBlocksPerSm / med;
    out->ms = ms;
    out->clk_mhz = (double)cyc[blocks - 1] / (ms * 1e-3) / 1e6;
    return Status::Ok();
}

}  // namespace
}  // namespace xk

extern "C" int xk_probe_pipes(xk_ctx* ctx, xk_pipe_peaks* out) {
    if (!ctx || !out) return XK_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = xk_pipe_peaks{};
    xk::DevBuf scratch;
    xk::ProbeRun f, m;
    // ~20-50 ms per probe at B200 clocks.
    const int fma_iters = 1 << 13, mufu_iters = 1 << 11;
    const double fma_ops = (double)fma_iters * 4 * xk::kProbeChains * 2 * xk::kProbeThreads;
    const double mufu_ops = (double)mufu_iters * 2 * xk::kProbeChains * xk::kProbeThreads;
    xk::Status st = xk::run_probe(xk::ffma2_probe, fma_iters, fma_ops, ctx->num_sms, ctx->stream,
                                  scratch, &f);
    if (st.ok())
        st = xk::run_probe(xk::mufu_probe, mufu_iters, mufu_ops, ctx->num_sms, ctx->stream,
                           scratch, &m);
    scratch.release();
    if (!st.ok()) {
        ctx->last_error = st.msg;
        return st.code;
    }
    out->fma_lane_ops_per_clk_sm = f.ops_per_clk_sm;
    out->mufu_ops_per_clk_sm = m.ops_per_clk_sm;
    out->fma_ms = f.ms;
    out->mufu_ms = m.ms;
    out->sm_clock_mhz = 0.5 * (f.clk_mhz + m.clk_mhz);
    out->num_sms = ctx->num_sms;
    return XK_OK;
}
