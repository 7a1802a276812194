// cpab_register.h -- launch descriptors of cpab_register.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cpab_internal.h"

namespace cpab {

struct LaunchCfg;

// Standalone remap (+ SSD) of N images [N, H, W] float32 through maps
// [N, H*W, 2] (float64 or float32); pixel coordinates px = x*sx + ox,
// py = y*sy + oy.
struct RemapArgs {
    const void *map;
    const float *src, *dst;   // dst == nullptr: remap only
    float *warped;            // may be nullptr when dst is given
    double *ll;               // [N] (with dst)
    double *partials;         // [N * tiles_per_image] workspace
    unsigned *tickets;        // [N] workspace, zero on entry
    int N, H, W, tile_px;
    double sx, ox, sy, oy, sigma;
};

// Fused registration likelihood for N instances, one image pair each.
struct RegisterArgs {
    Tess t;                   // 2D space
    const double *A, *T;      // [N, nC, 6] signed tables (sign -1: calc_T_inv)
    const float *src, *dst;   // [N, H, W]
    float *warped;            // [N, H, W] or nullptr
    double *ll;               // [N]
    double *partials;         // [N * tiles_per_image]
    unsigned *tickets;        // [N], zero on entry
    unsigned long long *counters;
    int N, H, W, tile_px;
    double sigma, dt;
    int nTimeSteps, nStepsODE;
    double h_sub;             // dt / nStepsODE, set on the host
    const volatile int *cancel;  // the context's cancel flag (device memory), polled between tiles, or nullptr
};

cudaError_t launch_remap_ssd(const RemapArgs &a, int map_prec, cudaStream_t s);
// Dynamic shared memory of k_register_ll: the tables and one double2 point slot per tile pixel.
size_t register_smem_bytes(int nC, int tile_px, int prec);
cudaError_t launch_register_ll(const RegisterArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s);

}  // namespace cpab
