// cpab_register3d.h -- launch descriptors of cpab_register3d.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cpab_internal.h"

namespace cpab {

struct LaunchCfg;

// Remap (+ SSD) of N volumes [N, H, W, D] float32 through maps [N, H*W*D, 3]
// (float64 or float32); voxel coordinates px = x*sx + ox, py = y*sy + oy,
// pz = z*sz + oz.
struct Remap3dArgs {
    const void *map;
    const float *src, *dst;   // dst == nullptr: remap only
    float *warped;            // may be nullptr when dst is given
    double *ll;               // [N] (with dst)
    double *partials;         // [N * tiles per volume] workspace
    unsigned *tickets;        // [N] workspace, zero on entry
    int N, H, W, D, tile_px;
    double sx, ox, sy, oy, sz, oz, sigma;
};

// Fused 3D registration likelihood for N instances, one volume pair each.
struct Register3dArgs {
    Tess t;                   // 3D space
    const double *A, *T;      // [N, nC, 12] signed tables (sign -1: calc_T_inv)
    const float *src, *dst;   // [N, H, W, D]
    float *warped;            // [N, H, W, D] or nullptr
    double *ll;               // [N]
    double *partials;
    unsigned *tickets;
    unsigned long long *counters;
    int N, H, W, D, tile_px;
    double sigma, dt;
    int nTimeSteps, nStepsODE;
    double h_sub;             // dt / nStepsODE, set on the host
    const volatile int *cancel;
};

size_t register3d_smem_bytes(int nC, int tile_px, int prec);
cudaError_t launch_remap3d_ssd(const Remap3dArgs &a, int map_prec, cudaStream_t s);
cudaError_t launch_register3d_ll(const Register3dArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s);

}  // namespace cpab
