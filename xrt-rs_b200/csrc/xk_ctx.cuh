// The context object behind the opaque xk_ctx handle (include/xk.h).
#pragma once

#include <string>

#include "xk_internal.cuh"
#include "xk_pr.cuh"

struct xk_ctx {
    int device = 0;
    int num_sms = 0;
    bool is_shared = false;
    std::string name;
    std::string last_error;
    std::mutex mu;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    xk::F64Workspace f64ws;
    xk::PrWorkspace prws;
    xk::PrOptions pr_opts;    // .tune points at `tune`
    xk::PrTuneCache tune;     // autotuned settings per bucket of solves
    double last_energy_ev = 0.0, last_dist_mm = 0.0;  // of the last planned F32PR solve
    xk::DevBuf in_rays, in_pix, out_field;
    xk::DevBuf in_beam;  // beam columns, normals and good indices (xk_beam_* calls)
    xk::FresnelWorkspace fresnel;
};
