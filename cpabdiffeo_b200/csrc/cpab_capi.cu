// cpab_capi.cu -- the extern "C" boundary declared in include/cpab_b200.h:
// argument validation, status codes and error strings, launch dispatch.
#include <cmath>
#include <new>

#include "cpab_ctx.h"

using namespace cpab;

thread_local char cpab::g_thread_err[512];

static size_t tables_smem(const cpab_ctx *c, int prec)
{
    // float64: A and T; float32: A and T - I
    return (size_t)c->t.nC * cell_len(c) * (prec == CPAB_F64 ? 2 * 8 : 2 * 4);
}

int cpab::max_smem_optin()
{
    static int v = 0;
    if (v == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 0)
            v = 227 * 1024;
    }
    return v;
}

extern "C" {

int cpab_ctx_create(cpab_ctx **out, int dim, int tess, const int *nCs, const double *incs)
{
    if (!out) return fail(nullptr, CPAB_BAD_ARG, "out is NULL");
    *out = nullptr;
    if (dim < 1 || dim > 3) return fail(nullptr, CPAB_BAD_ARG, "dim must be 1, 2 or 3 (got %d)", dim);
    if (tess != 1 && tess != 2) return fail(nullptr, CPAB_BAD_ARG, "tess must be 1 (I) or 2 (II) (got %d)", tess);
    if (dim == 1 && tess == 1)
        return fail(nullptr, CPAB_BAD_ARG, "1D spaces have type II tessellations only (cpab/cpaNd/_CpaSpace.py:77)");
    if (!nCs || !incs) return fail(nullptr, CPAB_BAD_ARG, "nCs/incs is NULL");
    cpab_ctx *c = new (std::nothrow) cpab_ctx();
    if (!c) return fail(nullptr, CPAB_NO_MEMORY, "out of host memory");
    if (!make_tess(dim, tess, nCs, incs, c->t)) {
        delete c;
        return fail(nullptr, CPAB_BAD_ARG, "invalid nCs/incs (need nCs >= 1, finite incs > 0, at most 2^20 cells)");
    }
    for (int k = 0; k < 3; ++k) c->nCs[k] = k < dim ? nCs[k] : 1;
    // cancel flag (only where a device is present)
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0 && cudaGetDevice(&c->device) == cudaSuccess) {
        void *d = nullptr, *h = nullptr;
        cudaStream_t st = nullptr;
        if (cudaMalloc(&d, sizeof(int)) == cudaSuccess && cudaHostAlloc(&h, 2 * sizeof(int), 0) == cudaSuccess &&
            cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
            static_cast<int *>(h)[0] = 0;
            static_cast<int *>(h)[1] = 1;
            if (cudaMemcpy(d, h, sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess) {
                c->cancel_dev = static_cast<int *>(d);
                c->cancel_src = static_cast<int *>(h);
                c->cancel_stream = st;
                d = h = nullptr;
                st = nullptr;
            }
        }
        if (d) cudaFree(d);
        if (h) cudaFreeHost(h);
        if (st) cudaStreamDestroy(st);
        if (!c->cancel_dev) c->device = -1;
        // facet tables of the 2D/3D exact scheme
        if (c->device >= 0 && dim >= 2) {
            std::vector<double> F;
            std::vector<int> nb;
            const int nF = build_facets(c->t, c->nCs, F, nb);
            void *fd = nullptr, *nd = nullptr;
            if (cudaMalloc(&fd, F.size() * sizeof(double)) == cudaSuccess &&
                cudaMalloc(&nd, nb.size() * sizeof(int)) == cudaSuccess &&
                cudaMemcpy(fd, F.data(), F.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
                cudaMemcpy(nd, nb.data(), nb.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess) {
                c->facets_dev = static_cast<double *>(fd);
                c->nbr_dev = static_cast<int *>(nd);
                c->nF = nF;
                fd = nd = nullptr;
            }
            if (fd) cudaFree(fd);
            if (nd) cudaFree(nd);
        }
    }
    cudaGetLastError();  // a missing device is not an error here
    *out = c;
    return CPAB_OK;
}

int cpab_ctx_destroy(cpab_ctx *ctx)
{
    if (ctx && ctx->cancel_dev) {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->cancel_stream);
        cudaStreamDestroy(ctx->cancel_stream);
        cudaFree(ctx->cancel_dev);
        cudaFreeHost(ctx->cancel_src);
        if (ctx->facets_dev) cudaFree(ctx->facets_dev);
        if (ctx->nbr_dev) cudaFree(ctx->nbr_dev);
        cudaSetDevice(prev);
    }
    delete ctx;
    return CPAB_OK;
}

// Write the device flag (0 or 1) and wait for that 4-byte copy only.
static int set_cancel_flag(cpab_ctx *ctx, int v)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (!ctx->cancel_dev) return fail(ctx, CPAB_UNSUPPORTED, "this context has no cancel flag");
    __atomic_store_n(&ctx->cancel_state, v, __ATOMIC_SEQ_CST);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != ctx->device) cudaSetDevice(ctx->device);
    cudaError_t e = cudaMemcpyAsync(ctx->cancel_dev, ctx->cancel_src + v, sizeof(int), cudaMemcpyHostToDevice,
                                    ctx->cancel_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->cancel_stream);
    if (prev != ctx->device) cudaSetDevice(prev);
    return cuda_status(ctx, e, "cancel flag");
}

int cpab_cancel(cpab_ctx *ctx) { return set_cancel_flag(ctx, 1); }

int cpab_clear_cancel(cpab_ctx *ctx) { return set_cancel_flag(ctx, 0); }

int cpab_cancel_requested(const cpab_ctx *ctx)
{
    return ctx ? __atomic_load_n(&ctx->cancel_state, __ATOMIC_SEQ_CST) : 0;
}

const char *cpab_last_error_string(const cpab_ctx *ctx) { return ctx ? ctx->err : g_thread_err; }

int cpab_ctx_num_cells(const cpab_ctx *ctx) { return ctx ? ctx->t.nC : -1; }
int cpab_ctx_cell_len(const cpab_ctx *ctx) { return ctx ? cell_len(ctx) : -1; }

int cpab_set_clamp(cpab_ctx *ctx, int enable, double lo, double hi)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (enable && !(lo <= hi)) return fail(ctx, CPAB_BAD_ARG, "clamp needs lo <= hi");
    ctx->clamp = enable ? 1 : 0;
    ctx->clamp_lo = lo;
    ctx->clamp_hi = hi;
    return CPAB_OK;
}

int cpab_set_launch(cpab_ctx *ctx, int block, int ctas_per_sm, int tile_pts)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (block && (block < 32 || block > 256 || block % 32))
        return fail(ctx, CPAB_BAD_ARG, "block must be a multiple of 32 in [32, 256] (got %d)", block);
    if (ctas_per_sm < 0 || ctas_per_sm > 64) return fail(ctx, CPAB_BAD_ARG, "ctas_per_sm out of range");
    if (tile_pts < 0 || tile_pts > 65536) return fail(ctx, CPAB_BAD_ARG, "tile_pts out of [1, 65536] (got %d)", tile_pts);
    if (block) ctx->cfg.block = block;
    if (ctas_per_sm) ctx->cfg.ctas_per_sm = ctas_per_sm;
    if (tile_pts) ctx->cfg.tile_pts = tile_pts;
    return CPAB_OK;
}

int cpab_set_max_ctas(cpab_ctx *ctx, int max_ctas)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (max_ctas < 0) return fail(ctx, CPAB_BAD_ARG, "max_ctas < 0");
    ctx->cfg.max_ctas = max_ctas;
    return CPAB_OK;
}

int cpab_set_cell_sort(cpab_ctx *ctx, int enable)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    ctx->cfg.sort = enable ? 1 : 0;
    return CPAB_OK;
}

int cpab_expm(cpab_ctx *ctx, const double *A, int N, double dt, int sign, double *signedA, double *Trels,
              void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (N < 0) return fail(ctx, CPAB_BAD_SHAPE, "N < 0");
    if (N == 0) return CPAB_OK;
    if (!A || !Trels) return fail(ctx, CPAB_BAD_ARG, "A/Trels is NULL");
    CPAB_CHECK_ALIGN(ctx, {A, 8, "A"}, {signedA, 8, "signedA"}, {Trels, 8, "Trels"});
    if (sign != 1 && sign != -1) return fail(ctx, CPAB_BAD_ARG, "sign must be +1 or -1");
    if (!std::isfinite(dt)) return fail(ctx, CPAB_BAD_ARG, "dt is not finite");
    return cuda_status(ctx, launch_expm(ctx->t.dim, A, signedA, Trels, (int64_t)N * ctx->t.nC, dt, (double)sign,
                                        (cudaStream_t)stream),
                       "expm launch");
}

int cpab_theta_to_trels(cpab_ctx *ctx, const double *B, int d, const double *theta, int N, double dt, int sign,
                        double *A, double *signedA, double *Trels, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (N < 0 || d < 1) return fail(ctx, CPAB_BAD_SHAPE, "need N >= 0 and d >= 1");
    if (N == 0) return CPAB_OK;
    if (!B || !theta || !Trels) return fail(ctx, CPAB_BAD_ARG, "B/theta/Trels is NULL");
    CPAB_CHECK_ALIGN(ctx, {B, 8, "B"}, {theta, 8, "theta"}, {A, 8, "A"}, {signedA, 8, "signedA"},
                     {Trels, 8, "Trels"});
    if (sign != 1 && sign != -1) return fail(ctx, CPAB_BAD_ARG, "sign must be +1 or -1");
    if (!std::isfinite(dt)) return fail(ctx, CPAB_BAD_ARG, "dt is not finite");
    return cuda_status(ctx, launch_theta_to_trels(ctx->t.dim, B, theta, d, ctx->t.nC, N, dt, (double)sign, A,
                                                  signedA, Trels, (cudaStream_t)stream),
                       "theta_to_trels launch");
}

int cpab_calc_cell_idx(cpab_ctx *ctx, const double *pts, int32_t *cell_idx, int64_t nPts, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (nPts < 0) return fail(ctx, CPAB_BAD_SHAPE, "nPts < 0");
    if (nPts == 0) return CPAB_OK;
    if (!pts || !cell_idx) return fail(ctx, CPAB_BAD_ARG, "pts/cell_idx is NULL");
    CPAB_CHECK_ALIGN(ctx, {pts, 8, "pts"}, {cell_idx, 4, "cell_idx"});
    return cuda_status(ctx, launch_cell_idx(ctx->t, pts, cell_idx, nPts, (cudaStream_t)stream), "cell_idx launch");
}

int cpab_calc_v(cpab_ctx *ctx, const double *A, const double *pts, double *vel, int64_t nPts, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (nPts < 0) return fail(ctx, CPAB_BAD_SHAPE, "nPts < 0");
    if (nPts == 0) return CPAB_OK;
    if (!A || !pts || !vel) return fail(ctx, CPAB_BAD_ARG, "A/pts/vel is NULL");
    CPAB_CHECK_ALIGN(ctx, {A, 8, "A"}, {pts, 8, "pts"}, {vel, 8, "vel"});
    size_t bytes = (size_t)nPts * ctx->t.dim * 8;
    if (overlaps(pts, bytes, vel, bytes)) return fail(ctx, CPAB_ALIAS, "pts and vel overlap");
    if ((size_t)ctx->t.nC * cell_len(ctx) * 8 > (size_t)max_smem_optin())
        return fail(ctx, CPAB_UNSUPPORTED, "cell table does not fit in shared memory");
    return cuda_status(ctx, launch_calc_v(ctx->t, A, pts, vel, nPts, (cudaStream_t)stream), "calc_v launch");
}

static int check_integrate(cpab_ctx *ctx, const double *signedA, const double *Trels, const void *pts, void *out,
                           int64_t nPts, int precision, int scheme, double dt, int nTimeSteps, int nStepsODE)
{
    if (precision != CPAB_F64 && precision != CPAB_F32)
        return fail(ctx, CPAB_BAD_DTYPE, "precision must be CPAB_F64 or CPAB_F32");
    if (scheme != CPAB_SCHEME_REF && scheme != CPAB_SCHEME_SIMPLE && scheme != CPAB_SCHEME_EXACT)
        return fail(ctx, CPAB_BAD_ARG, "unknown scheme %d", scheme);
    if (scheme == CPAB_SCHEME_EXACT && ctx->t.dim != 1 && !ctx->facets_dev)
        return fail(ctx, CPAB_UNSUPPORTED, "this context has no facet tables (created without a device)");
    if (scheme == CPAB_SCHEME_EXACT && ctx->t.dim != 1 && !Trels)
        return fail(ctx, CPAB_BAD_ARG, "Trels is NULL");
    if (nPts < 0) return fail(ctx, CPAB_BAD_SHAPE, "nPts < 0");
    if (nTimeSteps < 1) return fail(ctx, CPAB_BAD_ARG, "nTimeSteps must be >= 1");
    if (nStepsODE < 1) return fail(ctx, CPAB_BAD_ARG, "nStepsODE must be >= 1");
    if ((long long)nTimeSteps * nStepsODE > 0x7fffffffLL)
        return fail(ctx, CPAB_BAD_ARG, "nTimeSteps * nStepsODE overflows");
    if (!std::isfinite(dt)) return fail(ctx, CPAB_BAD_ARG, "dt is not finite");
    if (!signedA) return fail(ctx, CPAB_BAD_ARG, "signedA is NULL");
    if (scheme == CPAB_SCHEME_REF && !Trels) return fail(ctx, CPAB_BAD_ARG, "Trels is NULL");
    if (nPts > 0 && (!pts || !out)) return fail(ctx, CPAB_BAD_ARG, "pts/out is NULL");
    const size_t el = precision == CPAB_F64 ? 8 : 4;
    CPAB_CHECK_ALIGN(ctx, {signedA, 8, "signedA"}, {Trels, 8, "Trels"}, {pts, el, "pts"}, {out, el, "out"});
    size_t bytes = (size_t)nPts * ctx->t.dim * (precision == CPAB_F64 ? 8 : 4);
    if (nPts > 0 && overlaps(pts, bytes, out, bytes))
        return fail(ctx, CPAB_ALIAS, "pts and out cannot point to the same memory (_CpaCalcs.py:388)");
    size_t need;
    if (scheme == CPAB_SCHEME_EXACT && ctx->t.dim == 1) {
        need = exact1d_smem_bytes(ctx->t.nC, ctx->cfg.tile_pts, ctx->cfg.sort,
                                  precision == CPAB_F64 ? PREC_F64 : PREC_F32);
    } else {
        need = tables_smem(ctx, precision);
        if (ctx->cfg.sort) need += ((size_t)ctx->t.nC + 2 * (size_t)ctx->cfg.tile_pts) * sizeof(int);
    }
    if (need > (size_t)max_smem_optin())
        return fail(ctx, CPAB_UNSUPPORTED, "cell tables and tile scratch (%zu bytes) exceed shared memory", need);
    return CPAB_OK;
}

static IntegrateArgs make_args(cpab_ctx *ctx, const double *signedA, const double *Trels, const void *pts,
                               void *out, double dt, int nTimeSteps, int nStepsODE, uint64_t *counters)
{
    IntegrateArgs a;
    memset(&a, 0, sizeof(a));
    a.t = ctx->t;
    a.A = signedA;
    a.T = Trels;
    a.pts_in = pts;
    a.pts_out = out;
    a.dt = dt;
    a.nTimeSteps = nTimeSteps;
    a.nStepsODE = nStepsODE;
    a.h_sub = dt / (double)nStepsODE;
    a.clamp = ctx->clamp;
    a.clamp_lo = ctx->clamp_lo;
    a.clamp_hi = ctx->clamp_hi;
    a.counters = reinterpret_cast<unsigned long long *>(counters);
    a.max_crossings = 4 * ctx->t.nC + 8;
    a.sort = ctx->cfg.sort;
    a.cancel = cancel_ptr(ctx);
    a.facets = ctx->facets_dev;
    a.nbr = ctx->nbr_dev;
    a.nF = ctx->nF;
    return a;
}

static int run_integrate(cpab_ctx *ctx, IntegrateArgs &a, int precision, int scheme, int64_t uniform_tiles_total,
                         cudaStream_t s)
{
    LaunchCfg cfg = ctx->cfg;
    // small uniform launches: one CTA per tile (the persistent grid would leave CTAs idle)
    if (uniform_tiles_total > 0 && uniform_tiles_total < (int64_t)num_sms() * 2) cfg.grid = (int)uniform_tiles_total;
    if (cfg.grid > 0 && cfg.max_ctas > 0 && cfg.grid > cfg.max_ctas) cfg.grid = cfg.max_ctas;
    cudaError_t e = (scheme == CPAB_SCHEME_EXACT && a.t.dim == 1) ? launch_integrate_exact1d(a, precision, cfg, s)
                                                                   : launch_integrate(a, precision, scheme, cfg, s);
    return cuda_status(ctx, e, "integrate launch");
}

int cpab_calc_T(cpab_ctx *ctx, const double *signedA, const double *Trels, const void *pts, void *out,
                int64_t nPts, int precision, int scheme, double dt, int nTimeSteps, int nStepsODE,
                uint64_t *counters, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    int st = check_integrate(ctx, signedA, Trels, pts, out, nPts, precision, scheme, dt, nTimeSteps, nStepsODE);
    if (st != CPAB_OK) return st;
    CPAB_CHECK_ALIGN(ctx, {counters, 8, "counters"});
    if (nPts == 0) return CPAB_OK;
    IntegrateArgs a = make_args(ctx, signedA, Trels, pts, out, dt, nTimeSteps, nStepsODE, counters);
    a.batch.N = 1;
    a.batch.n_uniform = nPts;
    a.batch.offsets = nullptr;
    a.batch.tile_prefix = nullptr;
    a.batch.tile_pts = small_launch_tile(nPts, ctx->cfg.tile_pts);
    a.batch.tiles_per_inst = (nPts + a.batch.tile_pts - 1) / a.batch.tile_pts;
    return run_integrate(ctx, a, precision, scheme, a.batch.tiles_per_inst, (cudaStream_t)stream);
}

size_t cpab_batched_workspace_bytes(int N)
{
    if (N < 0) return 0;
    size_t b = (size_t)(N + 1) * sizeof(int64_t);
    return (b + 255) & ~(size_t)255;
}

int cpab_calc_T_batched(cpab_ctx *ctx, const double *signedA, const double *Trels, const void *pts, void *out,
                        int N, const int64_t *offsets, int64_t n_uniform, void *workspace, size_t workspace_bytes,
                        int precision, int scheme, double dt, int nTimeSteps, int nStepsODE, uint64_t *counters,
                        void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (N < 0) return fail(ctx, CPAB_BAD_SHAPE, "N < 0");
    if (N == 0) return CPAB_OK;
    if (!offsets && n_uniform < 0) return fail(ctx, CPAB_BAD_SHAPE, "n_uniform < 0");
    // Overlap is checked on the uniform extent only; ragged extents live on the device.
    int64_t nchk = offsets ? 0 : (int64_t)N * n_uniform;
    int st = check_integrate(ctx, signedA, Trels, pts, out, nchk, precision, scheme, dt, nTimeSteps, nStepsODE);
    if (st != CPAB_OK) return st;
    if (offsets && (!pts || !out)) return fail(ctx, CPAB_BAD_ARG, "pts/out is NULL");
    if (offsets && pts == out) return fail(ctx, CPAB_ALIAS, "pts and out are the same buffer");
    CPAB_CHECK_ALIGN(ctx, {offsets, 8, "offsets"}, {workspace, 8, "workspace"}, {counters, 8, "counters"});
    cudaStream_t s = (cudaStream_t)stream;
    IntegrateArgs a = make_args(ctx, signedA, Trels, pts, out, dt, nTimeSteps, nStepsODE, counters);
    a.batch.N = N;
    a.batch.tile_pts = ctx->cfg.tile_pts;
    int64_t uniform_tiles = 0;
    if (offsets) {
        if (!workspace || workspace_bytes < cpab_batched_workspace_bytes(N))
            return fail(ctx, CPAB_NO_MEMORY, "workspace of %zu bytes needed", cpab_batched_workspace_bytes(N));
        int64_t *prefix = static_cast<int64_t *>(workspace);
        cudaError_t e = launch_tile_prefix(offsets, prefix, N, a.batch.tile_pts, s);
        if (e != cudaSuccess) return cuda_status(ctx, e, "tile_prefix launch");
        a.batch.offsets = offsets;
        a.batch.tile_prefix = prefix;
    } else {
        if (n_uniform == 0) return CPAB_OK;
        a.batch.tile_pts = small_launch_tile((int64_t)N * n_uniform, ctx->cfg.tile_pts);
        a.batch.n_uniform = n_uniform;
        a.batch.tiles_per_inst = (n_uniform + a.batch.tile_pts - 1) / a.batch.tile_pts;
        uniform_tiles = a.batch.tiles_per_inst * N;
    }
    return run_integrate(ctx, a, precision, scheme, uniform_tiles, s);
}

int cpab_calc_trajectory(cpab_ctx *ctx, const double *signedA, const double *Trels, const double *pts, double *traj,
                         int64_t nPts, double dt, int nTimeSteps, int nStepsODE, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (!Trels) return fail(ctx, CPAB_BAD_ARG, "Trels is NULL");
    int st = check_integrate(ctx, signedA, Trels, pts, traj, 0, CPAB_F64, CPAB_SCHEME_REF, dt, nTimeSteps, nStepsODE);
    if (st != CPAB_OK) return st;
    if (nPts < 0) return fail(ctx, CPAB_BAD_SHAPE, "nPts < 0");
    if (nPts == 0) return CPAB_OK;
    if (!pts || !traj) return fail(ctx, CPAB_BAD_ARG, "pts/traj is NULL");
    CPAB_CHECK_ALIGN(ctx, {pts, 8, "pts"}, {traj, 8, "traj"});
    size_t in_bytes = (size_t)nPts * ctx->t.dim * 8, out_bytes = in_bytes * (size_t)(nTimeSteps + 1);
    if (overlaps(pts, in_bytes, traj, out_bytes)) return fail(ctx, CPAB_ALIAS, "pts and traj overlap");
    IntegrateArgs a = make_args(ctx, signedA, Trels, pts, traj, dt, nTimeSteps, nStepsODE, nullptr);
    return cuda_status(ctx, launch_trajectory(a, nPts, (cudaStream_t)stream), "trajectory launch");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free ragged batch (cpab_calc_T_batched_noalloc).
//
// Some callers cannot allocate device memory: a host application that owns
// the whole device pool and hands plugins only their inputs and outputs, or a
// latency-critical loop that must not pay for cudaMalloc's implicit
// synchronisation.  For them the tile bookkeeping of a ragged batch lives in
// this fixed array, compiled into the library.  Every GPU that loads the
// library holds it (CPAB_NOALLOC_MAX_INSTANCES + 1 int64 rounded up to 256
// bytes, about 512 KiB) until the
// process exits.  All calls share it and it keeps the last call's contents;
// each call rewrites every entry it reads, so nothing needs clearing, but two
// calls whose work overlaps on the GPU (different streams, or different host
// threads) race on it.  Host code must not pass the array's name to a kernel:
// outside device code that name is a host-side stand-in, not a device
// address.  The device address is looked up once per device, with that device
// current, on the first call made on it.
#include <mutex>

// Sized as cpab_batched_workspace_bytes(CPAB_NOALLOC_MAX_INSTANCES): (MAX + 1)
// int64 entries rounded up to 256 bytes, so a ragged call at exactly the
// maximum passes the workspace-size check of cpab_calc_T_batched.
constexpr size_t kNoallocScratchBytes = ((size_t)(CPAB_NOALLOC_MAX_INSTANCES + 1) * sizeof(int64_t) + 255) & ~(size_t)255;
static __device__ __align__(256) int64_t g_noalloc_tile_prefix[kNoallocScratchBytes / sizeof(int64_t)];

namespace {
constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
int64_t *g_noalloc_addr[kNoallocMaxDevices] = {nullptr};
}  // namespace

static int noalloc_scratch(cpab_ctx *ctx, int64_t **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(ctx, e, "cudaGetDevice");
    if (dev < 0 || dev >= kNoallocMaxDevices)
        return fail(ctx, CPAB_UNSUPPORTED, "device %d: the allocation-free entry point supports devices 0..%d", dev,
                    kNoallocMaxDevices - 1);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_tile_prefix);
        if (e != cudaSuccess) return cuda_status(ctx, e, "cudaGetSymbolAddress(g_noalloc_tile_prefix)");
        g_noalloc_addr[dev] = static_cast<int64_t *>(p);
    }
    *out = g_noalloc_addr[dev];
    return CPAB_OK;
}

extern "C" int cpab_calc_T_batched_noalloc(cpab_ctx *ctx, const double *signedA, const double *Trels,
                                           const void *pts, void *out, int N, const int64_t *offsets,
                                           int64_t n_uniform, int precision, int scheme, double dt,
                                           int nTimeSteps, int nStepsODE, uint64_t *counters, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (N > CPAB_NOALLOC_MAX_INSTANCES)
        return fail(ctx, CPAB_BAD_SHAPE,
                    "cpab_calc_T_batched_noalloc accepts at most %d instances (got %d); "
                    "use cpab_calc_T_batched with a workspace for larger batches",
                    CPAB_NOALLOC_MAX_INSTANCES, N);
    int64_t *scratch = nullptr;
    if (offsets && N > 0) {
        int st = noalloc_scratch(ctx, &scratch);
        if (st != CPAB_OK) return st;
    }
    return cpab_calc_T_batched(ctx, signedA, Trels, pts, out, N, offsets, n_uniform, scratch,
                               scratch ? sizeof(g_noalloc_tile_prefix) : 0, precision, scheme, dt, nTimeSteps,
                               nStepsODE, counters, stream);
}
