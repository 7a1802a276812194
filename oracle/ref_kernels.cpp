/*
 * ref_kernels.cpp -- host wrappers around the reference's calc_*.cu kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled once per (dimension, tessellation)
 * by oracle/Makefile with
 *   -DREF_DIM=<1|2|3> -DREF_TESS=<1|2> -DREF_SRC="<reference .cu path>"
 * The .cu file is included verbatim (cpab/gpu/calc_{1Dto1D,2Dto2D,3Dto3D}.cu,
 * the variant cpab/gpu/Calcs.py:100 selects for that dimension).
 *
 * Exported (C linkage), X = d<REF_DIM>_t<REF_TESS>:
 *   ref_X_calc_cell_idx, ref_X_calc_v, ref_X_calc_T, ref_X_calc_T_simple,
 *   ref_X_calc_trajectory
 * Argument lists follow the kernels (cpab/gpu/calc_2Dto2D.cu:323-602) plus the
 * cell count nC, which sets the emulated block size (the reference needs
 * blockDim >= N_CELLS for its shared-memory fill, cpab/gpu/Calcs.py:496-511).
 */
#include "ref_shim.h"
#include <omp.h>

#define N_CELLS 2048
#define DIM REF_DIM
#define TESS_TYPE REF_TESS

#define CAT3_(a, b, c) a##b##c
#define CAT3(a, b, c) CAT3_(a, b, c)
#define VNS CAT3(refns_d, REF_DIM, CAT3(_t, REF_TESS, ))
#define XNAME(f) CAT3(ref_d, REF_DIM, CAT3(_t, REF_TESS, _##f))

namespace VNS {
#include REF_SRC
}

/* Run kernel body `launch` over ceil(nPts/nC) emulated blocks of nC threads,
 * after a fill-only pass (block index past the data) on each host thread. */
#define EMULATE(nPts, nC, launch)                                              \
    do {                                                                       \
        const unsigned bd_ = (unsigned)(nC);                                   \
        const long nb_ = ((long)(nPts) + bd_ - 1) / bd_;                       \
        _Pragma("omp parallel")                                                \
        {                                                                      \
            blockDim = ref_dim3{bd_, 1, 1};                                    \
            blockIdx = ref_dim3{(unsigned)nb_, 0, 0};                          \
            for (unsigned t_ = 0; t_ < bd_; ++t_) {                            \
                threadIdx = ref_dim3{t_, 0, 0};                                \
                launch;                                                        \
            }                                                                  \
            _Pragma("omp for schedule(dynamic, 4)")                            \
            for (long b_ = 0; b_ < nb_; ++b_) {                                \
                blockIdx = ref_dim3{(unsigned)b_, 0, 0};                       \
                for (unsigned t_ = 0; t_ < bd_; ++t_) {                        \
                    threadIdx = ref_dim3{t_, 0, 0};                            \
                    launch;                                                    \
                }                                                              \
            }                                                                  \
        }                                                                      \
    } while (0)

extern "C" {

void XNAME(calc_cell_idx)(double *pts, int *cell_idx, int nPts, int nC0, int nC1, int nC2,
                          double ix, double iy, double iz, int nC)
{
    EMULATE(nPts, nC, VNS::calc_cell_idx(pts, cell_idx, nPts, nC0, nC1, nC2, ix, iy, iz));
}

void XNAME(calc_v)(double *pts, double *vel, double *As, int nPts, int nC0, int nC1, int nC2,
                   double ix, double iy, double iz, int nC)
{
    EMULATE(nPts, nC, VNS::calc_v(pts, vel, As, nPts, nC0, nC1, nC2, ix, iy, iz));
}

void XNAME(calc_T)(const double *pos0, double *pos, const double *Trels, const double *As,
                   double dt, int nTimeSteps, int nStepsOdeSolver, int nPts,
                   int nC0, int nC1, int nC2, double ix, double iy, double iz, int nC)
{
    EMULATE(nPts, nC, VNS::calc_T(pos0, pos, Trels, As, dt, nTimeSteps, nStepsOdeSolver,
                                  nPts, nC0, nC1, nC2, ix, iy, iz));
}

void XNAME(calc_T_simple)(const double *pos0, double *pos, const double *As,
                          double dt, int nTimeSteps, int nStepsOdeSolver, int nPts,
                          int nC0, int nC1, int nC2, double ix, double iy, double iz, int nC)
{
    EMULATE(nPts, nC, VNS::calc_T_simple(pos0, pos, As, dt, nTimeSteps, nStepsOdeSolver,
                                         nPts, nC0, nC1, nC2, ix, iy, iz));
}

/* pos: [nTimeSteps * nPts, DIM]; rows [0, nPts) hold the start points on
 * entry (cpab/gpu/Calcs.py:771-773). */
void XNAME(calc_trajectory)(double *pos, const double *Trels, const double *As,
                            double dt, int nTimeSteps, int nStepsOdeSolver, int nPts,
                            int nC0, int nC1, int nC2, double ix, double iy, double iz, int nC)
{
    EMULATE(nPts, nC, VNS::calc_trajectory(pos, Trels, As, dt, nTimeSteps, nStepsOdeSolver,
                                           nPts, nC0, nC1, nC2, ix, iy, iz));
}

}  // extern "C"
