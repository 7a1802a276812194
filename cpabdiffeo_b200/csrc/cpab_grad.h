// cpab_grad.h -- launch descriptor of cpab_grad.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cpab_internal.h"

namespace cpab {

struct GradArgs {
    Tess t;
    const double *A;         // [N, nC, ne] signed matrices of the forward map
    const double *T;         // [N, nC, ne] their closed-form steps expm(dt A) (reference scheme)
    const double *pts;       // [N * n, DIM] start points
    const double *grad_out;  // [N * n, DIM] dLoss/dT(x)
    double *out;             // [N * n, DIM] T(x) or nullptr
    double *grad_in;         // [N * n, DIM] dLoss/dx or nullptr
    double *gA;              // [N, nC, ne] dLoss/d(signed A), accumulated (zero on entry)
    double *gT;              // [N, nC, ne] dLoss/dT scratch, zero on entry (reference scheme)
    double *gS;              // [N, nC, ne] dLoss/d(sub-step map) scratch, zero on entry (FP32 reference scheme)
    double *ckpt;            // [ceil(nT/ck), N * n, DIM] scratch (FP32: [.., 2 * DIM] floats, hi and lo)
    double h_sub;            // dt / nStepsODE
    int N;
    int64_t n_per_inst;
    double dt;
    int nTimeSteps, nStepsODE, ck;
};

cudaError_t launch_grad_simple(const GradArgs &a, cudaStream_t s);
cudaError_t launch_grad_ref(const GradArgs &a, cudaStream_t s);
cudaError_t launch_grad_ref_f32(const GradArgs &a, cudaStream_t s);
cudaError_t launch_bt_times(const double *B, const double *G, double *out, int DA, int d, int N, double scale,
                            cudaStream_t s);

}  // namespace cpab
