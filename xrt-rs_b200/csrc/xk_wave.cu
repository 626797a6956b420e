// The two producers in front of the Kirchhoff path, on the device:
//
//   prepare_wave             (src/waves/prepare_wave.rs:40-68)  screen grid
//   beam_to_diffraction_rays (src/waves/prepare_wave.rs:78-111) beam -> rays
//
// Both are O(N + M) gathers, bound by HBM (a few bytes per output double);
// they exist so that a beam's columns are uploaded once and the ray records
// and the screen are built where the solve reads them. Every floating-point
// step is an explicitly rounded intrinsic in the reference's order (no FMA
// contraction), so the outputs equal the reference's bit for bit.

#include <algorithm>

#include "xk_internal.cuh"

namespace xk {
namespace {

constexpr int kThreads = 256;

// Reference: frac = i / (n - 1) - 0.5 when n > 1, else 0 (prepare_wave.rs:44-48,54-58).
__device__ __forceinline__ double grid_frac(size_t i, size_t n) {
    if (n <= 1) return 0.0;
    return __dsub_rn(__ddiv_rn((double)i, (double)(n - 1)), 0.5);
}

__global__ void __launch_bounds__(kThreads) wave_kernel(WaveGrid g, double* __restrict__ x,
                                                        double* __restrict__ y,
                                                        double* __restrict__ z) {
    const size_t total = g.nx * g.nz;
    for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < total;
         i += (size_t)gridDim.x * kThreads) {
        const size_t ix = i / g.nz, iz = i - ix * g.nz;
        // center + frac * 2.0 * d, evaluated left to right (prepare_wave.rs:49,59).
        x[i] = __dadd_rn(g.cx, __dmul_rn(__dmul_rn(grid_frac(ix, g.nx), 2.0), g.dx));
        y[i] = g.cy;
        z[i] = __dadd_rn(g.cz, __dmul_rn(__dmul_rn(grid_frac(iz, g.nz), 2.0), g.dz));
    }
}

struct RayCols {
    double* c[12];
};

__global__ void __launch_bounds__(kThreads) beam_rays_kernel(BeamDev b,
                                                             const uint64_t* __restrict__ good,
                                                             size_t n_good, RayCols out) {
    for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n_good;
         i += (size_t)gridDim.x * kThreads) {
        const uint64_t j = good[i];
        const double n0 = b.normals[3 * j], n1 = b.normals[3 * j + 1], n2 = b.normals[3 * j + 2];
        const double a = b.a[j], bb = b.b[j], c = b.c[j];
        // nl = n[0]*a + n[1]*b + n[2]*c (prepare_wave.rs:89), left to right.
        const double nl = __dadd_rn(__dadd_rn(__dmul_rn(n0, a), __dmul_rn(n1, bb)), __dmul_rn(n2, c));
        out.c[0][i] = b.x[j];
        out.c[1][i] = b.y[j];
        out.c[2][i] = b.z[j];
        out.c[3][i] = n0;
        out.c[4][i] = n1;
        out.c[5][i] = n2;
        out.c[6][i] = nl;
        if (b.es_re) {
            out.c[7][i] = b.es_re[j];
            out.c[8][i] = b.es_im[j];
            out.c[9][i] = b.ep_re[j];
            out.c[10][i] = b.ep_im[j];
        } else {  // no amplitudes: es = 1, ep = 0 (prepare_wave.rs:91-97)
            out.c[7][i] = 1.0;
            out.c[8][i] = 0.0;
            out.c[9][i] = 0.0;
            out.c[10][i] = 0.0;
        }
        out.c[11][i] = b.e[j];
    }
}

int grid_for(size_t n) {
    // Grid-stride loops; a few waves of 256-thread blocks over 148 SMs cover
    // any size without a per-element block.
    const size_t blocks = (n + kThreads - 1) / kThreads;
    return (int)std::min<size_t>(blocks, 148 * 16);
}

}  // namespace

Status wave_enqueue(const WaveGrid& g, double* x, double* y, double* z, cudaStream_t stream) {
    const size_t total = g.nx * g.nz;
    if (total == 0) return Status::Ok();
    wave_kernel<<<grid_for(total), kThreads, 0, stream>>>(g, x, y, z);
    XK_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

Status beam_rays_enqueue(const BeamDev& beam, const uint64_t* good, size_t n_good,
                         double* const out[12], cudaStream_t stream) {
    if (n_good == 0) return Status::Ok();
    RayCols cols;
    for (int f = 0; f < 12; ++f) cols.c[f] = out[f];
    beam_rays_kernel<<<grid_for(n_good), kThreads, 0, stream>>>(beam, good, n_good, cols);
    XK_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

namespace {

__global__ void __launch_bounds__(kThreads)
    gpu_records_kernel(const xk_gpu_ray* __restrict__ rays, size_t n,
                       const xk_gpu_pixel* __restrict__ pix, size_t m, RayCols cols, double* px,
                       double* py, double* pz) {
    const size_t stride = (size_t)gridDim.x * kThreads;
    for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n; i += stride) {
        const xk_gpu_ray r = rays[i];
        // GpuRay order x, y, z, nx, ny, nz, nl, energy, es, ep -> RaysDev order.
        const float v[12] = {r.x, r.y, r.z, r.nx, r.ny, r.nz, r.nl,
                             r.es_re, r.es_im, r.ep_re, r.ep_im, r.energy};
#pragma unroll
        for (int f = 0; f < 12; ++f) cols.c[f][i] = (double)v[f];
    }
    for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < m; i += stride) {
        const xk_gpu_pixel p = pix[i];
        px[i] = (double)p.x;
        py[i] = (double)p.y;
        pz[i] = (double)p.z;
    }
}

__global__ void __launch_bounds__(kThreads) interleave_kernel(FieldDev f, size_t m,
                                                              double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < m;
         i += (size_t)gridDim.x * kThreads)
        reinterpret_cast<double4*>(out)[i] = make_double4(f.es_re[i], f.es_im[i], f.ep_re[i],
                                                          f.ep_im[i]);
}

}  // namespace

Status gpu_records_enqueue(const xk_gpu_ray* rays, size_t n, const xk_gpu_pixel* pix, size_t m,
                           double* const ray_cols[12], double* px, double* py, double* pz,
                           cudaStream_t stream) {
    if (n == 0 && m == 0) return Status::Ok();
    RayCols cols;
    for (int f = 0; f < 12; ++f) cols.c[f] = ray_cols[f];
    gpu_records_kernel<<<grid_for(std::max(n, m)), kThreads, 0, stream>>>(rays, n, pix, m, cols,
                                                                          px, py, pz);
    XK_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

Status interleave_field_enqueue(const FieldDev& f, size_t m, double* out, cudaStream_t stream) {
    if (m == 0) return Status::Ok();
    interleave_kernel<<<grid_for(m), kThreads, 0, stream>>>(f, m, out);
    XK_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

}  // namespace xk
