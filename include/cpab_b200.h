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
 *  CPAB_SCHEME_EXACT  the flow across cell boundaries with hitting times.
 *                     1D: closed form (cpab/cpa1d/calcs/ClosedFormInt.py:
 *                     64-256).  2D/3D (no reference counterpart; replaces
 *                     the midpoint fallback of calc_2Dto2D.cu:167-197):
 *                     REF's closed-form steps and keep test; a step that
 *                     leaves its cell is re-integrated in nStepsODE
 *                     sub-steps of the exact flow expm(h*A_c), and a
 *                     sub-step whose end leaves the cell moves to the
 *                     facet at its hitting time and on in the neighbour.
 *                     Hitting times in FP64 in both precisions. */
enum { CPAB_SCHEME_REF = 0, CPAB_SCHEME_SIMPLE = 1, CPAB_SCHEME_EXACT = 2 };

/* Counter slots written by calls that take `counters` (uint64[CPAB_CNT_N],
 * added to): closed-form steps kept (cell visits for the 1D exact scheme),
 * fallback steps, sub-steps, points finished, points that hit the crossing
 * cap (2D/3D exact: sub-steps whose exit no interior facet explained),
 * points with a NaN result, CTAs stopped by cpab_cancel, facet crossings
 * resolved at their hitting time (2D/3D exact). */
enum { CPAB_CNT_FAST = 0, CPAB_CNT_FALLBACK = 1, CPAB_CNT_SUBSTEPS = 2, CPAB_CNT_POINTS = 3,
       CPAB_CNT_FAILED = 4, CPAB_CNT_NAN = 5, CPAB_CNT_CANCELLED = 6, CPAB_CNT_CROSSINGS = 7,
       CPAB_CNT_N = 8 };

/* ------------------------------------------------------------------ context */

/* Create a context for one tessellation of [xmins, xmaxs] on the current
 * device.  dim in {1,2,3}; tess 1 = type I (triangles in 2D, 5 tetrahedra
 * per box in 3D), 2 = type II (boxes; the only type in 1D).  nCs[dim] boxes
 * per axis; incs[dim] box sizes exactly as the reference derives them
 * (cpab/cpaNd/_CpaSpace.py:278-294).  Replaces the per-space kernel JIT
 * (cpab/gpu/Calcs.py:66-203, N_CELLS/DIM/TESS_TYPE macros :159-162). */
int cpab_ctx_create(cpab_ctx **out, int dim, int tess, const int *nCs_host, const double *incs_host);
/* Facet tables of a tessellation (host only; no device needed): per cell,
 * n_facets rows (outward unit normal, -offset) -- g(x) = n.x - offset <= 0
 * inside -- in facets[nC * n_facets * (dim+1)], and the cell across each
 * facet (-1 on the domain boundary) in nbr[nC * n_facets].  Simplex facet k
 * is opposite vertex k of the reference's vertex order
 * (cpab/cpa2d/Tessellation.py:73-138, cpab/cpa3d/Tessellation.py:62-200);
 * box facets are (x_lo, x_hi, y_lo, y_hi, z_lo, z_hi).  facets/nbr may be
 * NULL to query n_facets.  The tables the 2D/3D exact scheme uses; no
 * counterpart in the reference. */
int cpab_tess_facets(int dim, int tess, const int *nCs_host, const double *incs_host, double *facets, int *nbr,
                     int *n_facets);
int cpab_ctx_destroy(cpab_ctx *ctx);
/* Last error of this context (or of the calling thread when ctx == NULL). */
const char *cpab_last_error_string(const cpab_ctx *ctx);
/* Number of cells and length of one cell's matrix (dim*(dim+1)). */
int cpab_ctx_num_cells(const cpab_ctx *ctx);
int cpab_ctx_cell_len(const cpab_ctx *ctx);

/* Cancellation.  Each context owns a flag in device memory (on the device
 * current at cpab_ctx_create) that the persistent integration, exact,
 * registration and landmark kernels read every 8th tile; once it is set they
 * finish the tile in hand, skip the rest and count themselves in
 * CPAB_CNT_CANCELLED (no device fault, no trap).  cpab_cancel /
 * cpab_clear_cancel write the flag with a 4-byte copy on the context's own
 * stream (the copy engine, so no SM is needed while kernels occupy the GPU)
 * and return once it has landed; they may be called from any host thread
 * while a launch runs.  The flag stays set until cpab_clear_cancel.
 * CPAB_UNSUPPORTED if the context has no flag (it is created with the context
 * when a device is present).  No counterpart in the reference (its launches
 * cannot be stopped). */
int cpab_cancel(cpab_ctx *ctx);
int cpab_clear_cancel(cpab_ctx *ctx);
int cpab_cancel_requested(const cpab_ctx *ctx);

/* 1D zero-velocity boundary epilogue: clamp outputs of calc_T to [lo, hi]
 * (threshold_krnl, cpab/cpaNd/_CpaSpace.py:35-43 and :655-664). */
int cpab_set_clamp(cpab_ctx *ctx, int enable, double lo, double hi);

/* Launch shape of the integration kernel: threads per CTA (32..256, a
 * multiple of 32), resident CTAs per SM of the persistent grid, points per
 * CTA tile.  0 keeps the current value.  Used by the autotuner. */
int cpab_set_launch(cpab_ctx *ctx, int block, int ctas_per_sm, int tile_pts);

/* Cell-sort the points of each CTA tile by start cell before integrating
 * (REF / SIMPLE schemes): lanes of a warp then share cells (shared-memory
 * broadcasts, coherent branches).  Results are unchanged (every point is
 * integrated on its own).  Off by default; the autotuner decides.  No
 * reference counterpart (the reference launches one thread per point in input
 * order, cpab/gpu/Calcs.py:515). */
/* Cap every persistent launch of this context (integration, exact,
 * registration and landmark kernels) at max_ctas CTAs (0 = no cap), leaving
 * the other SMs to kernels of other streams -- a server keeps long
 * registration jobs from occupying every SM while transform batches wait.
 * Results do not depend on the cap.  No counterpart in the reference. */
int cpab_set_max_ctas(cpab_ctx *ctx, int max_ctas);
int cpab_set_cell_sort(cpab_ctx *ctx, int enable);

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

/* ------------------------------------------------------------------ images */

/* Scratch bytes of cpab_remap_ssd for N images of H x W. */
size_t cpab_remap_workspace_bytes(int N, int H, int W);

/* Bilinear remap of N float32 images src [N, H, W] through maps [N, H*W, 2]
 * (x, y per pixel; float64 or float32 per map_precision), with cv2.remap
 * semantics -- x is the column, y the row, integer coordinates at pixel
 * centres, taps outside the image read 0 (the remap of
 * cpab/cpa2d/TransformWrapper.py:261-317, remap_fwd / remap_inv).  A map point
 * (x, y) is sampled at pixel coordinates (x*sx + ox, y*sy + oy): (W, -0.5, H,
 * -0.5) for points of the unit square, (1, 0, 1, 0) for pixel units.
 * warped [N, H, W] float32 may be NULL when dst is given.  With dst [N, H, W]
 * the same pass computes the Gaussian log-likelihood
 *   ll[n] = sum_i -0.5 (warped_i - dst_i)^2 / sigma^2
 * (cpab/cpa2d/model/transformations/register/gpu/gaussian.py:15-34 and the
 * reduction of _ScaleDependentLogLikelihoodGeneral.py:108-131) in a fixed
 * order (identical alone or batched).  workspace: cpab_remap_workspace_bytes.
 * ctx may be NULL (errors then go to the thread's error string). */
int cpab_remap_ssd(cpab_ctx *ctx, const void *map, int map_precision, const float *src, const float *dst,
                   int N, int H, int W, double sx, double ox, double sy, double oy, double sigma,
                   float *warped, double *ll, void *workspace, size_t workspace_bytes, void *stream);

/* Scratch bytes of cpab_register_ll for N image pairs of H x W. */
size_t cpab_register_workspace_bytes(const cpab_ctx *ctx, int N, int H, int W);

/* The registration log-likelihood of N (theta, src, dst) triples in one
 * launch (ScaleDependentLogLikelihoodGaussian.calc_ll,
 * cpab/cpa2d/model/transformations/register/_ScaleDependentLogLikelihoodGaussian.py:34-109):
 * every pixel centre ((c+0.5)/W, (r+0.5)/H) of the unit square is integrated
 * with instance n's tables (pass sign -1 tables for calc_T_inv, as the
 * reference does), src[n] is sampled there (bilinear, as cpab_remap_ssd) and
 * compared with dst[n]; ll[n] as in cpab_remap_ssd.  The transformed points
 * are never written.  2D spaces; REF scheme; precision sets the integration
 * arithmetic (CPAB_F64 bit-exact).  warped may be NULL. */
int cpab_register_ll(cpab_ctx *ctx, const double *signedA, const double *Trels, int N, const float *src,
                     const float *dst, int H, int W, double sigma, int precision, double dt, int nTimeSteps,
                     int nStepsODE, double *ll, float *warped, void *workspace, size_t workspace_bytes,
                     uint64_t *counters, void *stream);

/* Scratch bytes of cpab_remap3d_ssd for N volumes of H x W x D (needed with dst). */
size_t cpab_remap3d_workspace_bytes(int N, int H, int W, int D);

/* Trilinear remap of N float32 volumes [N, H, W, D] (remap3d of the external
 * of.gpu.remap, called from remap_fwd / remap_inv at
 * cpab/cpa3d/TransformWrapper.py:230-286).  Volumes are indexed
 * [row][col][slice], the order of the reference's dense 3D grid
 * (np.mgrid[0:Ny, 0:Nx, 0:Nz], cpab/cpa3d/calcs/_CpaCalcs.py:45-76); a map
 * point (x, y, z) = (column, row, slice) is sampled at voxel coordinates
 * (x*sx + ox, y*sy + oy, z*sz + oz), integer coordinates at voxel centres,
 * taps outside the volume read 0.  map [N, H*W*D, 3] float64 or float32.
 * With dst the same pass gives ll[n] = sum -0.5 (warped - dst)^2 / sigma^2 in
 * a fixed order; warped may then be NULL. */
int cpab_remap3d_ssd(cpab_ctx *ctx, const void *map, int map_precision, const float *src, const float *dst,
                     int N, int H, int W, int D, double sx, double ox, double sy, double oy, double sz, double oz,
                     double sigma, float *warped, double *ll, void *workspace, size_t workspace_bytes,
                     void *stream);

/* Scratch bytes of cpab_register3d_ll. */
size_t cpab_register3d_workspace_bytes(const cpab_ctx *ctx, int N, int H, int W, int D);

/* The registration log-likelihood of N (theta, src, dst) volume triples in
 * one launch: the 3D form of cpab_register_ll (the reference's registration
 * likelihood, cpab/cpa2d/model/transformations/register/
 * _ScaleDependentLogLikelihoodGaussian.py:34-109, exists for 2D images; the
 * 3D remap it would use is remap3d above).  Every voxel centre
 * ((c+0.5)/W, (r+0.5)/H, (k+0.5)/D) of the unit cube is integrated with
 * instance n's tables (sign -1 for calc_T_inv), src[n] is sampled there
 * (trilinear) and compared with dst[n].  3D spaces; REF scheme. */
int cpab_register3d_ll(cpab_ctx *ctx, const double *signedA, const double *Trels, int N, const float *src,
                       const float *dst, int H, int W, int D, double sigma, int precision, double dt,
                       int nTimeSteps, int nStepsODE, double *ll, float *warped, void *workspace,
                       size_t workspace_bytes, uint64_t *counters, void *stream);

/* Scratch bytes of cpab_landmark_ll for N instances of n_lm landmarks. */
size_t cpab_landmark_workspace_bytes(const cpab_ctx *ctx, int N, int n_lm);

/* The Gaussian landmark log-likelihood of N instances in one launch
 * (ScaleDependentLogLikelihoodGaussian.calc_ll of
 * cpab/cpa2d/model/transformations/landmarks/_ScaleDependentLogLikelihoodGaussian.py:29-73
 * with calc_err_per_sample / calc_ll_per_sample of its gpu/gaussian.py:12-22;
 * 1D: cpab/cpa1d/model/transformations/landmarks/, same formula):
 *   ll[n] = sum_i -0.5 |T_n(src_i) - dst_i|^2 / sigma^2,
 * T_n = calc_T_fwd with instance n's tables (REF scheme), any dimension and
 * tessellation.  src / dst are float64 [*, n_lm, dim]; instance n reads its
 * landmarks at src + n * src_stride * dim (src_stride 0: one set shared by
 * all instances; likewise dst).  The sum is taken in a fixed order (the
 * reference's __call__ then divides by n_lm in 2D).  transformed
 * [N, n_lm, dim] float64 receives T_n(src_i) unless NULL.  precision sets the
 * integration arithmetic (CPAB_F64: the transformed points are bit-exact). */
int cpab_landmark_ll(cpab_ctx *ctx, const double *signedA, const double *Trels, int N, const double *src,
                     int64_t src_stride, const double *dst, int64_t dst_stride, int n_lm, double sigma,
                     int precision, double dt, int nTimeSteps, int nStepsODE, double *ll, double *transformed,
                     void *workspace, size_t workspace_bytes, uint64_t *counters, void *stream);

/* ------------------------------------------------------------------ inference */

/* Random-walk proposals for C chains (Proposal.__call__,
 * cpab/cpaNd/inference/Proposal.py:29-64, diagonal covariance :61-64):
 *   theta_prop[c] = theta[c] + scale * prop_std .* z,  z ~ N(0, I)
 * z from Philox4x32-10 keyed by seed with counter (chain, *step, 0, pair),
 * Box-Muller in double.  step: device int64 read by the kernel. */
int cpab_mcmc_propose(cpab_ctx *ctx, int C, int d, const double *theta, const double *prop_std, double scale,
                      uint64_t seed, const int64_t *step, double *theta_prop, void *stream);

/* Local proposals for C chains (the use_local branch of Proposal.__call__,
 * cpab/cpaNd/inference/Proposal.py:65-130): with velTess the velocities at the
 * tessellation's nV vertices, pick a vertex k uniformly (Philox stream 2,
 * counter (chain, *step, 2, 0)), add s * z to its velocity (z ~ N(0, I_dim),
 * counters (chain, *step, 2, 1 + pair)) -- or set it to 0 when bdry[k] (the
 * reference's boundary rule, :104-120) -- and map the change to theta:
 *   theta_prop[c] = theta[c] + G[k] dv,   v_k = E[k] theta.
 * E [nV, dim, d], G [nV, d, dim] float64 and bdry [nV] int32 come from the
 * space's geometry (local_proposal_tables in cpabdiffeo_b200/space.py); the
 * reference's s is scale_local_proposal * min(XMAXS) (0.01 in 1D).  Simplicial
 * tessellations (1D, type I), as in the reference. */
int cpab_mcmc_propose_local(cpab_ctx *ctx, int C, int d, const double *theta, int nV, const double *E,
                            const double *G, const int32_t *bdry, double s, uint64_t seed, const int64_t *step,
                            double *theta_prop, void *stream);

/* Accept/reject for C chains and advance *step by one (Metropolis.step,
 * cpab/cpaNd/inference/Metropolis.py:41-85): log_ratio = (ll_prop - ll) *
 * inv_npts (+ wlp * (lp' - lp) with the prior precision prior_prec [d, d]);
 * accept when log_ratio > 0, else with u ~ U(0,1) (Philox stream 1):
 * rule 0 accepts when log(u) > log_ratio -- the reference's own test
 * (Metropolis.py:77-82) -- and rule 1 when log(u) < log_ratio (textbook MH).
 * On accept theta, ll (and lp) take the proposal's values and n_accepted
 * (may be NULL) counts it. */
int cpab_mcmc_accept(cpab_ctx *ctx, int C, int d, double *theta, const double *theta_prop, double *ll,
                     const double *ll_prop, double inv_npts, const double *prior_prec, double wlp, double *lp,
                     int rule, uint64_t seed, int64_t *step, int64_t *n_accepted, void *stream);

/* Scratch bytes of cpab_mcmc_run (256-byte aligned workspace). */
size_t cpab_mcmc_run_workspace_bytes(const cpab_ctx *ctx, int C, int d, int H, int W);

/* n_steps Metropolis steps of C image-registration chains in one call
 * (Metropolis.run, cpab/cpaNd/inference/Metropolis.py:41-85, with the
 * random-walk Proposal.py:29-64 and the registration likelihood of
 * cpab_register_ll): ll[c] is first set to the likelihood of theta[c], then
 * every step enqueues cpab_mcmc_propose, cpab_theta_to_trels (sign -1),
 * cpab_register_ll and cpab_mcmc_accept on `stream` -- the same kernels in the
 * same order as a caller stepping one call at a time, so the chains are
 * identical.  theta [C, d], ll [C], *step and n_accepted (may be NULL) are
 * updated in place on the device; B [D, d] is the space's basis; no prior.
 * 2D spaces.  Asynchronous: returns after enqueueing. */
int cpab_mcmc_run(cpab_ctx *ctx, const double *B, int d, int C, double *theta, const double *prop_std, double scale,
                  const float *src, const float *dst, int H, int W, double sigma, int precision, double dt,
                  int nTimeSteps, int nStepsODE, double inv_npts, int rule, uint64_t seed, int64_t *step,
                  int n_steps, double *ll, int64_t *n_accepted, void *workspace, size_t workspace_bytes,
                  void *stream);

/* ------------------------------------------------------------------ gradient */

/* Scratch bytes of cpab_grad_theta: checkpoints every ck time steps. */
size_t cpab_grad_workspace_bytes(const cpab_ctx *ctx, int N, int64_t n_per_inst, int nTimeSteps, int ck);

/* Gradient of a scalar loss of T(x) through the midpoint scheme
 * (calc_T_simple semantics: nTimeSteps * nStepsODE sub-steps, the scheme whose
 * derivative the reference's unbound calc_grad_theta carries forward,
 * cpab/gpu/calc_2Dto2D.cu:202-319,448-491, cpab/cpaNd/_CpaSpace.py:669-686).
 * N instances of n_per_inst points (pts, grad_out = dLoss/dT(x): [N*n, dim]
 * float64); signedA [N, nC, ne] = sign * A.  Runs the forward again (out, may
 * be NULL, receives T(x)), then the discrete adjoint backwards:
 *   gA [N, nC*ne]      dLoss/d(signedA) (written; no accumulation across calls)
 *   dtheta [N, d]      sign * B^T gA (NULL to skip; needs B [nC*ne, d])
 *   grad_pts [N*n, dim] dLoss/dx (NULL to skip).
 * ck: checkpoint stride in time steps (1 = fastest, nTimeSteps = least
 * memory); workspace: cpab_grad_workspace_bytes.  nStepsODE <= 256. */
int cpab_grad_theta(cpab_ctx *ctx, const double *B, int d, const double *signedA, int N, const double *pts,
                    int64_t n_per_inst, const double *grad_out, double dt, int nTimeSteps, int nStepsODE, int sign,
                    int ck, double *out, double *grad_pts, double *gA, double *dtheta, void *workspace,
                    size_t workspace_bytes, void *stream);

/* Scratch bytes of cpab_grad_theta_ref: checkpoints every ck time steps plus
 * two per-cell sums [N, nC, ne] (dLoss/dTrels, dLoss/d(sub-step map)). */
size_t cpab_grad_ref_workspace_bytes(const cpab_ctx *ctx, int N, int64_t n_per_inst, int nTimeSteps, int ck);

/* Gradient of a scalar loss of T(x) through the reference scheme (calc_T:
 * per time step the closed-form step with Trels = expm(dt * signedA) when its
 * end point stays in the cell, else nStepsODE midpoint sub-steps;
 * cpab/gpu/calc_2Dto2D.cu:348-408, cpab/cpaNd/_CpaSpace.py:626-667, whose
 * sensitivity code, calc_grad_theta :669-686, is never bound).  Same
 * arguments and outputs as cpab_grad_theta plus Trels [N, nC, ne] from the
 * same signedA and dt (cpab_theta_to_trels) and `precision`: pts, grad_out,
 * out and grad_pts are float64 (CPAB_F64) or float32 (CPAB_F32); signedA,
 * Trels, gA and dtheta are float64 either way.  The forward run again here is
 * calc_T's arithmetic in that precision (out: T(x), bit for bit); the
 * adjoint follows the forward's branch at every step (closed-form step or
 * fallback, and every sub-step's cell) and maps the per-cell dLoss/dTrels to
 * dLoss/dA through the adjoint Frechet derivative of expm (FP32: also the
 * sub-steps' per-cell map).  Workspace: cpab_grad_ref_workspace_bytes.
 * nStepsODE <= 256. */
int cpab_grad_theta_ref(cpab_ctx *ctx, const double *B, int d, const double *signedA, const double *Trels, int N,
                        const void *pts, int64_t n_per_inst, const void *grad_out, int precision, double dt,
                        int nTimeSteps, int nStepsODE, int sign, int ck, void *out, void *grad_pts, double *gA,
                        double *dtheta, void *workspace, size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CPAB_B200_H */
