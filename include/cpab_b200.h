/*
 * cpab_b200.h -- C ABI of libcpab_b200.so, the sm_100a CPAB transform
 * library.  Plain pointers, sizes and a CUDA stream: no C++ or torch types.
 *
 * Every entry point replaces one step of the reference's Python/pycuda
 * path (freifeld/cpabDiffeo; file:line below).  A Python binding is
 * cpabdiffeo_b200/_lib.py (ctypes); the CpaSpace / TransformWrapper mirror
 * above it keeps the reference's method names.
 *
 * Conventions
 *  - All array arguments are DEVICE pointers owned by the caller, unless the
 *    name ends in _host.  The library never frees them.
 *  - Points are row-major [nPts, dim] (the reference's C-contiguous layout,
 *    cpab/gpu/Calcs.py:940-945); float64 (CPAB_F64) or float32 (CPAB_F32).
 *  - Per-cell matrices are row-major dim x (dim+1) ("As_vectorized",
 *    cpab/cpaNd/_CpaCalcs.py:126-128), float64, [N, nC, dim*(dim+1)] for a
 *    batch of N transforms.
 *  - stream: a cudaStream_t (NULL = legacy default stream).  Calls are
 *    asynchronous; nothing synchronises except where stated.
 *  - Every call returns a cpab_status.  On failure nothing was launched and
 *    cpab_last_error_string() describes the problem.  No call traps or
 *    asserts on the device.
 *  - A context is not thread-safe: use one per host thread (or serialise).
 */
#ifndef CPAB_B200_H
#define CPAB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cpab_ctx cpab_ctx;

typedef enum {
    CPAB_OK = 0,
    CPAB_BAD_ARG = 1,       /* invalid scalar argument (dim, tess, steps, ...)      */
    CPAB_BAD_SHAPE = 2,     /* sizes inconsistent with the space                     */
    CPAB_BAD_DTYPE = 3,     /* unsupported precision                                 */
    CPAB_ALIAS = 4,         /* input and output overlap (_CpaCalcs.py:382-389)      */
    CPAB_NO_MEMORY = 5,     /* workspace too small / allocation failed               */
    CPAB_CANCELLED = 6,     /* cpab_cancel() was called                              */
    CPAB_TIMEOUT = 7,       /* a bounded wait or iteration cap ran out               */
    CPAB_NUMERIC = 8,       /* NaN/inf detected where the call checks                */
    CPAB_CUDA_ERROR = 9,    /* a CUDA runtime call failed                            */
    CPAB_UNSUPPORTED = 10   /* configuration not built                               */
} cpab_status;

enum { CPAB_F64 = 0, CPAB_F32 = 1 };

/* Integration schemes.
 *  CPAB_SCHEME_REF    calc_T: per time step Trel = expm(dt*A_c) applied in
 *                     closed form, kept if the end point stays in the cell,
 *                     else nStepsODE explicit-midpoint sub-steps
 *                     (cpab/gpu/calc_2Dto2D.cu:348-408).  Bit-exact to the
 *                     reference's double arithmetic in CPAB_F64.
 *  CPAB_SCHEME_SIMPLE calc_T_simple: midpoint sub-steps only
 *                     (cpab/gpu/calc_2Dto2D.cu:412-445).
 *  CPAB_SCHEME_EXACT  closed-form flow with cell-boundary hitting times
 *                     (1D; cpab/cpa1d/calcs/ClosedFormInt.py:64-256). */
enum { CPAB_SCHEME_REF = 0, CPAB_SCHEME_SIMPLE = 1, CPAB_SCHEME_EXACT = 2 };

/* Counter slots written by calls that take `counters` (uint64[5], added to). */
enum { CPAB_CNT_FAST = 0, CPAB_CNT_FALLBACK = 1, CPAB_CNT_SUBSTEPS = 2, CPAB_CNT_POINTS = 3,
       CPAB_CNT_FAILED = 4, CPAB_CNT_N = 5 };

/* ------------------------------------------------------------------ context */

/* Create a context for one tessellation of [xmins, xmaxs] on the current
 * device.  dim in {1,2,3}; tess 1 = type I (triangles in 2D, 5 tetrahedra
 * per box in 3D), 2 = type II (boxes; the only type in 1D).  nCs[dim] boxes
 * per axis; incs[dim] box sizes exactly as the reference derives them
 * (cpab/cpaNd/_CpaSpace.py:278-294).  Replaces the per-space kernel JIT
 * (cpab/gpu/Calcs.py:66-203, N_CELLS/DIM/TESS_TYPE macros :159-162). */
int cpab_ctx_create(cpab_ctx **out, int dim, int tess, const int *nCs_host, const double *incs_host);
int cpab_ctx_destroy(cpab_ctx *ctx);
/* Last error of this context (or of the calling thread when ctx == NULL). */
const char *cpab_last_error_string(const cpab_ctx *ctx);
/* Number of cells and length of one cell's matrix (dim*(dim+1)). */
int cpab_ctx_num_cells(const cpab_ctx *ctx);
int cpab_ctx_cell_len(const cpab_ctx *ctx);

/* 1D zero-velocity boundary epilogue: clamp outputs of calc_T to [lo, hi]
 * (threshold_krnl, cpab/cpaNd/_CpaSpace.py:35-43 and :655-664). */
int cpab_set_clamp(cpab_ctx *ctx, int enable, double lo, double hi);

/* Launch shape of the integration kernel: threads per CTA (32..256, a
 * multiple of 32), resident CTAs per SM of the persistent grid, points per
 * CTA tile.  0 keeps the current value.  Used by the autotuner. */
int cpab_set_launch(cpab_ctx *ctx, int block, int ctas_per_sm, int tile_pts);

/* ------------------------------------------------------------------ prologue */

/* Per-cell signed matrices and their exponentials for N transforms:
 *   signedA = sign * A,  Trels = expm(dt * sign * A)
 * (prepare_signedSqAs_and_Tlocals_for_gpu, cpab/cpaNd/_CpaCalcs.py:227-372;
 * 1D closed form :272-294; 2D gpu_expm cpab/gpu/expm/expm_affine_by_series_2D.py:246;
 * 3D gpu_expm expm_affine_by_series_3D.py:228).  A: [N, nC, ne].
 * signedA may be NULL. */
int cpab_expm(cpab_ctx *ctx, const double *A, int N, double dt, int sign,
              double *signedA, double *Trels, void *stream);

/* A = B . theta for N thetas fused with cpab_expm: theta [N, d] row-major,
 * B [nC*ne, d] row-major (the basis of the CPA space).  A (may be NULL)
 * receives [N, nC*ne].  Replaces CpaSpace.theta2Avees + update_pat
 * (cpab/cpaNd/_CpaSpace.py:366-376, _PAT.py:48-59) and the expm prologue. */
int cpab_theta_to_trels(cpab_ctx *ctx, const double *B, int d, const double *theta, int N,
                        double dt, int sign, double *A, double *signedA, double *Trels, void *stream);

/* ------------------------------------------------------------------ per point */

/* int32 cell index of each point (calc_cell_idx, cpab/gpu/calc_2Dto2D.cu:323-344;
 * host cpab/cpaNd/_CpaCalcs.py:59-88).  pts float64. */
int cpab_calc_cell_idx(cpab_ctx *ctx, const double *pts, int32_t *cell_idx, int64_t nPts, void *stream);

/* Velocity v = A_c [x; 1] (calc_v, cpab/gpu/calc_2Dto2D.cu:561-602; host
 * cpab/cpaNd/_CpaCalcs.py:95-165).  A: [nC, ne] of one transform, float64. */
int cpab_calc_v(cpab_ctx *ctx, const double *A, const double *pts, double *vel, int64_t nPts, void *stream);

/* T(x) for one transform (calc_T / calc_T_simple, cpab/gpu/Calcs.py:339-624;
 * host cpab/cpaNd/_CpaCalcs.py:376-743; sign dispatch
 * cpab/cpaNd/_CpaSpace.py:626-667).  signedA, Trels: [nC, ne] from
 * cpab_expm with the same dt and sign (Trels unused by CPAB_SCHEME_SIMPLE).
 * pts/out: [nPts, dim] in `precision`; must not overlap (CPAB_ALIAS).
 * counters: uint64[CPAB_CNT_N] device array or NULL. */
int cpab_calc_T(cpab_ctx *ctx, const double *signedA, const double *Trels,
                const void *pts, void *out, int64_t nPts, int precision, int scheme,
                double dt, int nTimeSteps, int nStepsODE, uint64_t *counters, void *stream);

/* Scratch bytes cpab_calc_T_batched needs for N ragged instances. */
size_t cpab_batched_workspace_bytes(int N);

/* T(x) for N transforms in one persistent launch.  Instance i uses tables
 * signedA[i], Trels[i] ([N, nC, ne]) and the points
 *   [offsets[i], offsets[i+1])          if offsets (device int64[N+1]) != NULL,
 *   [i*n_uniform, (i+1)*n_uniform)      otherwise.
 * workspace: device scratch of cpab_batched_workspace_bytes(N) bytes (ragged
 * batches only; may be NULL when offsets == NULL).  No reference
 * counterpart beyond calling calc_T once per theta. */
int cpab_calc_T_batched(cpab_ctx *ctx, const double *signedA, const double *Trels,
                        const void *pts, void *out, int N, const int64_t *offsets, int64_t n_uniform,
                        void *workspace, size_t workspace_bytes, int precision, int scheme,
                        double dt, int nTimeSteps, int nStepsODE, uint64_t *counters, void *stream);

/* Largest N cpab_calc_T_batched_noalloc accepts. */
#define CPAB_NOALLOC_MAX_INSTANCES 65536

/* cpab_calc_T_batched without caller scratch: for callers that cannot
 * allocate device memory (a host that owns the whole device pool and gives a
 * plugin only its inputs and outputs, or a latency-critical loop that must not
 * pay for cudaMalloc's implicit synchronisation).  The ragged-batch
 * bookkeeping lives in a fixed device array inside the library (512 KiB per
 * GPU that loads it, held until exit), so N is limited to
 * CPAB_NOALLOC_MAX_INSTANCES (larger N -> CPAB_BAD_SHAPE).  Makes no
 * allocation.  The first call on a device looks up the array's device
 * address with that device current; make that first call before any stream
 * capture.  Calls share the array: calls whose work overlaps on the GPU
 * (other streams, other threads) race.  No counterpart in the reference. */
int cpab_calc_T_batched_noalloc(cpab_ctx *ctx, const double *signedA, const double *Trels,
                                const void *pts, void *out, int N, const int64_t *offsets, int64_t n_uniform,
                                int precision, int scheme, double dt, int nTimeSteps, int nStepsODE,
                                uint64_t *counters, void *stream);

/* Trajectories (calc_trajectory, cpab/gpu/calc_2Dto2D.cu:499-556; host
 * cpab/cpaNd/_CpaCalcs.py:795-871): traj [(nTimeSteps+1), nPts, dim]
 * float64, row 0 = pts.  The reference supports 2D only; all dims here. */
int cpab_calc_trajectory(cpab_ctx *ctx, const double *signedA, const double *Trels,
                         const double *pts, double *traj, int64_t nPts,
                         double dt, int nTimeSteps, int nStepsODE, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CPAB_B200_H */
