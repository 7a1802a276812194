// cpab_landmarks.h -- launch descriptor of cpab_landmarks.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cpab_internal.h"

namespace cpab {

struct LaunchCfg;

// Gaussian landmark log-likelihood of N instances.
struct LandmarkArgs {
    Tess t;
    const double *A, *T;      // [N, nC, ne] signed tables (sign +1: calc_T_fwd)
    const double *src, *dst;  // landmarks [*, n_lm, dim]
    int64_t src_stride;       // points between instances' landmark sets (0: one set shared by all)
    int64_t dst_stride;
    double *transformed;      // [N, n_lm, dim] or nullptr
    double *ll;               // [N]
    double *partials;         // [N * tiles per instance] workspace
    unsigned *tickets;        // [N] workspace, zero on entry
    unsigned long long *counters;
    int N, n_lm, tile_pts;
    double sigma, dt;
    int nTimeSteps, nStepsODE;
    double h_sub;             // dt / nStepsODE, set on the host
    int clamp;                // the context's end-point clamp (1D zero boundary), as calc_T
    double clamp_lo, clamp_hi;
    const volatile int *cancel;
};

size_t landmark_smem_bytes(const Tess &t, int tile_pts, int prec);
cudaError_t launch_landmark_ll(const LandmarkArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s);

}  // namespace cpab
