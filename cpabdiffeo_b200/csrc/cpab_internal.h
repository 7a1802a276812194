// cpab_internal.h -- launch descriptors shared by the kernels and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cpab_cell.cuh"

namespace cpab {

enum Precision { PREC_F64 = 0, PREC_F32 = 1 };

// Integration schemes.
//  REF    : calc_T of cpab/gpu/calc_2Dto2D.cu:348-408 -- per time step a
//           closed-form step with Trel = expm(dt*A_c), kept when the end
//           point is still in the start cell, else nStepsODE midpoint steps.
//  SIMPLE : calc_T_simple, calc_2Dto2D.cu:412-445 -- midpoint steps only.
//  EXACT  : the flow across cell boundaries with hitting times.  1D:
//           cpab/cpa1d/calcs/ClosedFormInt.py:64-256 restated (k_exact1d).
//           2D/3D: REF's closed-form steps and keep test; a step that
//           leaves its cell is re-integrated in nStepsODE sub-steps of the
//           exact flow S_c = expm(h A_c), a sub-step whose end leaves the
//           cell resolved at the facet hitting times (exact_substep_cross).
enum Scheme { SCHEME_REF = 0, SCHEME_SIMPLE = 1, SCHEME_EXACT = 2 };

// A batch of N independent transforms ("instances"), each with its own
// cell tables and its own point range.  Uniform batches have n_uniform
// points per instance; ragged batches give device offsets[N+1].
struct Batch {
    int N;
    int64_t n_uniform;
    const int64_t *offsets;      // [N+1] or nullptr
    const int64_t *tile_prefix;  // [N+1] tiles per instance (prefix) or nullptr
    int64_t tiles_per_inst;      // uniform batches
    int tile_pts;                // points per CTA tile
};

struct IntegrateArgs {
    Tess t;
    const double *A;      // [N, nC, ne] signed velocity matrices
    const double *T;      // [N, nC, ne] Trel = expm(dt * signed A)  (REF)
    const void *pts_in;   // [nPts, DIM] float64 or float32
    void *pts_out;        // same layout
    Batch batch;
    double dt;
    int nTimeSteps;
    int nStepsODE;
    double h_sub;         // dt / nStepsODE, set on the host (read from parameter space, not a register)
    int clamp;            // 1D zero-velocity boundary: clamp to [lo, hi]
    double clamp_lo, clamp_hi;
    unsigned long long *counters;  // [CNT_N] or nullptr (slots below)
    int max_crossings;    // EXACT: give up after this many boundary crossings
    int sort;             // REF/SIMPLE: process each tile's points in order of their start cell
    const volatile int *cancel;  // the context's cancel flag (device memory), polled between tiles, or nullptr
    const double *facets; // EXACT 2D/3D: [nC, nF, DIM+1] (outward unit normal, -offset) per cell facet
    const int *nbr;       // EXACT 2D/3D: [nC, nF] cell across each facet, -1 on the domain boundary
    int nF;               // facets per cell
};

// Counters slots.
// CNT_NAN: points whose result has a NaN coordinate; CNT_CANCELLED: CTAs that
// stopped early because the context's cancel flag was set.
// CNT_CROSSINGS: EXACT 2D/3D facet crossings resolved at their hitting time
// (CNT_FAILED there: sub-steps whose exit no interior facet explained).
enum { CNT_FAST = 0, CNT_FALLBACK = 1, CNT_SUBSTEPS = 2, CNT_POINTS = 3, CNT_FAILED = 4, CNT_NAN = 5,
       CNT_CANCELLED = 6, CNT_CROSSINGS = 7, CNT_N = 8 };

// Facet tables of a tessellation (cpab_facets.cu).
int facets_per_cell(const Tess &t);

}  // namespace cpab
