// cpab_capi_register.cu -- C ABI of the remap / registration-likelihood
// kernels (declared in include/cpab_b200.h).
#include <cmath>

#include "cpab_ctx.h"
#include "cpab_landmarks.h"
#include "cpab_reduce.cuh"
#include "cpab_register.h"
#include "cpab_register3d.h"

using namespace cpab;

namespace {

constexpr int kRemapTilePx = 2048;

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct WsLayout {
    size_t partials_off, tickets_off, total;
};

WsLayout ws_layout(int N, int64_t tiles_per_image)
{
    WsLayout w;
    w.partials_off = 0;
    w.tickets_off = align256((size_t)N * (size_t)tiles_per_image * sizeof(double));
    w.total = w.tickets_off + align256((size_t)N * sizeof(unsigned));
    return w;
}

int64_t tiles_of(int H, int W, int tile_px) { return ((int64_t)H * W + tile_px - 1) / tile_px; }

// Tile of the fused likelihood kernels over `total` pixels (voxels): the
// small-launch rule rounded up to whole 256-point sum chunks.  Their sums do
// not depend on the tile (finish_tile_chunks), so the tile may follow the
// launch size.
int likelihood_tile(int64_t total, int tile_pts)
{
    const int t = small_launch_tile(total, tile_pts);
    return (t + kSumChunk - 1) / kSumChunk * kSumChunk;
}

int check_images(cpab_ctx *ctx, int N, int H, int W)
{
    if (N < 0) return fail(ctx, CPAB_BAD_SHAPE, "N < 0");
    if (H < 1 || W < 1) return fail(ctx, CPAB_BAD_SHAPE, "image size %d x %d", H, W);
    if ((int64_t)H * W > (int64_t)1 << 31) return fail(ctx, CPAB_BAD_SHAPE, "image too large");
    return CPAB_OK;
}

}  // namespace

extern "C" {

size_t cpab_remap_workspace_bytes(int N, int H, int W)
{
    if (N < 0 || H < 1 || W < 1) return 0;
    return ws_layout(N, tiles_of(H, W, kRemapTilePx)).total;
}

int cpab_remap_ssd(cpab_ctx *ctx, const void *map, int map_precision, const float *src, const float *dst, int N,
                   int H, int W, double sx, double ox, double sy, double oy, double sigma, float *warped,
                   double *ll, void *workspace, size_t workspace_bytes, void *stream)
{
    int st = check_images(ctx, N, H, W);
    if (st != CPAB_OK) return st;
    if (N == 0) return CPAB_OK;
    if (map_precision != CPAB_F64 && map_precision != CPAB_F32)
        return fail(ctx, CPAB_BAD_DTYPE, "map precision must be CPAB_F64 or CPAB_F32");
    if (!map || !src) return fail(ctx, CPAB_BAD_ARG, "map/src is NULL");
    if (!dst && !warped) return fail(ctx, CPAB_BAD_ARG, "nothing to compute: dst and warped are both NULL");
    if (dst && !ll) return fail(ctx, CPAB_BAD_ARG, "ll is NULL (needed with dst)");
    if (dst && !(sigma > 0) ) return fail(ctx, CPAB_BAD_ARG, "sigma must be positive");
    if (!std::isfinite(sx) || !std::isfinite(ox) || !std::isfinite(sy) || !std::isfinite(oy))
        return fail(ctx, CPAB_BAD_ARG, "pixel mapping is not finite");
    CPAB_CHECK_ALIGN(ctx, {map, map_precision == CPAB_F64 ? 8u : 4u, "map"}, {src, 4, "src"}, {dst, 4, "dst"},
                     {warped, 4, "warped"}, {ll, 8, "ll"}, {workspace, 8, "workspace"});
    const int64_t tpi = tiles_of(H, W, kRemapTilePx);
    const WsLayout L = ws_layout(N, tpi);
    RemapArgs a;
    memset(&a, 0, sizeof(a));
    a.map = map;
    a.src = src;
    a.dst = dst;
    a.warped = warped;
    a.ll = ll;
    a.N = N;
    a.H = H;
    a.W = W;
    a.tile_px = kRemapTilePx;
    a.sx = sx;
    a.ox = ox;
    a.sy = sy;
    a.oy = oy;
    a.sigma = dst ? sigma : 1.0;
    cudaStream_t s = (cudaStream_t)stream;
    if (dst) {
        if (!workspace || workspace_bytes < L.total)
            return fail(ctx, CPAB_NO_MEMORY, "workspace of %zu bytes needed", L.total);
        char *w = static_cast<char *>(workspace);
        a.partials = reinterpret_cast<double *>(w + L.partials_off);
        a.tickets = reinterpret_cast<unsigned *>(w + L.tickets_off);
        cudaError_t e = cudaMemsetAsync(a.tickets, 0, (size_t)N * sizeof(unsigned), s);
        if (e != cudaSuccess) return cuda_status(ctx, e, "ticket reset");
    }
    return cuda_status(ctx, launch_remap_ssd(a, map_precision == CPAB_F64 ? PREC_F64 : PREC_F32, s),
                       "remap_ssd launch");
}

size_t cpab_register_workspace_bytes(const cpab_ctx *ctx, int N, int H, int W)
{
    if (!ctx || N < 0 || H < 1 || W < 1) return 0;
    return ws_layout(N, tiles_of(H, W, kSumChunk)).total;  // one partial per 256-pixel chunk
}

int cpab_register_ll(cpab_ctx *ctx, const double *signedA, const double *Trels, int N, const float *src,
                     const float *dst, int H, int W, double sigma, int precision, double dt, int nTimeSteps,
                     int nStepsODE, double *ll, float *warped, void *workspace, size_t workspace_bytes,
                     uint64_t *counters, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (ctx->t.dim != 2) return fail(ctx, CPAB_UNSUPPORTED, "the registration likelihood is built for 2D spaces");
    int st = check_images(ctx, N, H, W);
    if (st != CPAB_OK) return st;
    if (N == 0) return CPAB_OK;
    if (precision != CPAB_F64 && precision != CPAB_F32)
        return fail(ctx, CPAB_BAD_DTYPE, "precision must be CPAB_F64 or CPAB_F32");
    if (!signedA || !Trels || !src || !dst || !ll) return fail(ctx, CPAB_BAD_ARG, "NULL argument");
    CPAB_CHECK_ALIGN(ctx, {signedA, 8, "signedA"}, {Trels, 8, "Trels"}, {src, 4, "src"}, {dst, 4, "dst"},
                     {ll, 8, "ll"}, {warped, 4, "warped"}, {workspace, 8, "workspace"}, {counters, 8, "counters"});
    if (!(sigma > 0)) return fail(ctx, CPAB_BAD_ARG, "sigma must be positive");
    if (nTimeSteps < 1 || nStepsODE < 1) return fail(ctx, CPAB_BAD_ARG, "nTimeSteps and nStepsODE must be >= 1");
    if (!std::isfinite(dt)) return fail(ctx, CPAB_BAD_ARG, "dt is not finite");
    const int tile_px = likelihood_tile((int64_t)N * H * W, ctx->cfg.tile_pts);
    // cell tables plus one point slot per pixel of a tile
    if (register_smem_bytes(ctx->t.nC, tile_px, precision == CPAB_F64 ? PREC_F64 : PREC_F32) >
        (size_t)max_smem_optin())
        return fail(ctx, CPAB_UNSUPPORTED, "cell tables and tile scratch exceed shared memory");
    const WsLayout L = ws_layout(N, tiles_of(H, W, kSumChunk));
    if (!workspace || workspace_bytes < L.total)
        return fail(ctx, CPAB_NO_MEMORY, "workspace of %zu bytes needed", L.total);
    RegisterArgs a;
    memset(&a, 0, sizeof(a));
    a.t = ctx->t;
    a.A = signedA;
    a.T = Trels;
    a.src = src;
    a.dst = dst;
    a.warped = warped;
    a.ll = ll;
    char *w = static_cast<char *>(workspace);
    a.partials = reinterpret_cast<double *>(w + L.partials_off);
    a.tickets = reinterpret_cast<unsigned *>(w + L.tickets_off);
    a.counters = reinterpret_cast<unsigned long long *>(counters);
    a.N = N;
    a.H = H;
    a.W = W;
    a.tile_px = tile_px;
    a.sigma = sigma;
    a.dt = dt;
    a.nTimeSteps = nTimeSteps;
    a.nStepsODE = nStepsODE;
    a.h_sub = dt / (double)nStepsODE;
    a.cancel = cancel_ptr(ctx);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(a.tickets, 0, (size_t)N * sizeof(unsigned), s);
    if (e != cudaSuccess) return cuda_status(ctx, e, "ticket reset");
    return cuda_status(ctx, launch_register_ll(a, precision == CPAB_F64 ? PREC_F64 : PREC_F32, ctx->cfg, s),
                       "register_ll launch");
}

static int check_volumes(cpab_ctx *ctx, int N, int H, int W, int D)
{
    if (N < 0) return fail(ctx, CPAB_BAD_SHAPE, "N < 0");
    if (H < 1 || W < 1 || D < 1) return fail(ctx, CPAB_BAD_SHAPE, "volume size %d x %d x %d", H, W, D);
    if ((int64_t)H * W * D > (int64_t)1 << 31) return fail(ctx, CPAB_BAD_SHAPE, "volume too large");
    return CPAB_OK;
}

static int64_t tiles_of3(int H, int W, int D, int tile_px)
{
    return ((int64_t)H * W * D + tile_px - 1) / tile_px;
}

size_t cpab_remap3d_workspace_bytes(int N, int H, int W, int D)
{
    if (N < 0 || H < 1 || W < 1 || D < 1) return 0;
    return ws_layout(N, tiles_of3(H, W, D, kRemapTilePx)).total;
}

int cpab_remap3d_ssd(cpab_ctx *ctx, const void *map, int map_precision, const float *src, const float *dst, int N,
                     int H, int W, int D, double sx, double ox, double sy, double oy, double sz, double oz,
                     double sigma, float *warped, double *ll, void *workspace, size_t workspace_bytes, void *stream)
{
    int st = check_volumes(ctx, N, H, W, D);
    if (st != CPAB_OK) return st;
    if (N == 0) return CPAB_OK;
    if (map_precision != CPAB_F64 && map_precision != CPAB_F32)
        return fail(ctx, CPAB_BAD_DTYPE, "map precision must be CPAB_F64 or CPAB_F32");
    if (!map || !src) return fail(ctx, CPAB_BAD_ARG, "map/src is NULL");
    if (!dst && !warped) return fail(ctx, CPAB_BAD_ARG, "nothing to compute: dst and warped are both NULL");
    if (dst && !ll) return fail(ctx, CPAB_BAD_ARG, "ll is NULL (needed with dst)");
    if (dst && !(sigma > 0)) return fail(ctx, CPAB_BAD_ARG, "sigma must be positive");
    if (!std::isfinite(sx) || !std::isfinite(ox) || !std::isfinite(sy) || !std::isfinite(oy) || !std::isfinite(sz) ||
        !std::isfinite(oz))
        return fail(ctx, CPAB_BAD_ARG, "voxel mapping is not finite");
    CPAB_CHECK_ALIGN(ctx, {map, map_precision == CPAB_F64 ? 8u : 4u, "map"}, {src, 4, "src"}, {dst, 4, "dst"},
                     {warped, 4, "warped"}, {ll, 8, "ll"}, {workspace, 8, "workspace"});
    const WsLayout L = ws_layout(N, tiles_of3(H, W, D, kRemapTilePx));
    if (dst && (!workspace || workspace_bytes < L.total))
        return fail(ctx, CPAB_NO_MEMORY, "workspace of %zu bytes needed", L.total);
    Remap3dArgs a;
    memset(&a, 0, sizeof(a));
    a.map = map;
    a.src = src;
    a.dst = dst;
    a.warped = warped;
    a.ll = ll;
    a.N = N;
    a.H = H;
    a.W = W;
    a.D = D;
    a.tile_px = kRemapTilePx;
    a.sx = sx;
    a.ox = ox;
    a.sy = sy;
    a.oy = oy;
    a.sz = sz;
    a.oz = oz;
    a.sigma = sigma;
    cudaStream_t s = (cudaStream_t)stream;
    if (dst) {
        char *w = static_cast<char *>(workspace);
        a.partials = reinterpret_cast<double *>(w + L.partials_off);
        a.tickets = reinterpret_cast<unsigned *>(w + L.tickets_off);
        cudaError_t e = cudaMemsetAsync(a.tickets, 0, (size_t)N * sizeof(unsigned), s);
        if (e != cudaSuccess) return cuda_status(ctx, e, "ticket reset");
    }
    return cuda_status(ctx, launch_remap3d_ssd(a, map_precision == CPAB_F64 ? PREC_F64 : PREC_F32, s),
                       "remap3d launch");
}

size_t cpab_register3d_workspace_bytes(const cpab_ctx *ctx, int N, int H, int W, int D)
{
    if (!ctx || N < 0 || H < 1 || W < 1 || D < 1) return 0;
    return ws_layout(N, tiles_of3(H, W, D, kSumChunk)).total;  // one partial per 256-voxel chunk
}

int cpab_register3d_ll(cpab_ctx *ctx, const double *signedA, const double *Trels, int N, const float *src,
                       const float *dst, int H, int W, int D, double sigma, int precision, double dt, int nTimeSteps,
                       int nStepsODE, double *ll, float *warped, void *workspace, size_t workspace_bytes,
                       uint64_t *counters, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (ctx->t.dim != 3) return fail(ctx, CPAB_UNSUPPORTED, "the 3D registration likelihood needs a 3D space");
    int st = check_volumes(ctx, N, H, W, D);
    if (st != CPAB_OK) return st;
    if (N == 0) return CPAB_OK;
    if (precision != CPAB_F64 && precision != CPAB_F32)
        return fail(ctx, CPAB_BAD_DTYPE, "precision must be CPAB_F64 or CPAB_F32");
    if (!signedA || !Trels || !src || !dst || !ll) return fail(ctx, CPAB_BAD_ARG, "NULL argument");
    if (!(sigma > 0)) return fail(ctx, CPAB_BAD_ARG, "sigma must be positive");
    if (nTimeSteps < 1 || nStepsODE < 1) return fail(ctx, CPAB_BAD_ARG, "nTimeSteps and nStepsODE must be >= 1");
    if ((long long)nTimeSteps * nStepsODE > 0x7fffffffLL)
        return fail(ctx, CPAB_BAD_ARG, "nTimeSteps * nStepsODE overflows");
    if (!std::isfinite(dt)) return fail(ctx, CPAB_BAD_ARG, "dt is not finite");
    CPAB_CHECK_ALIGN(ctx, {signedA, 8, "signedA"}, {Trels, 8, "Trels"}, {src, 4, "src"}, {dst, 4, "dst"},
                     {ll, 8, "ll"}, {warped, 4, "warped"}, {workspace, 8, "workspace"}, {counters, 8, "counters"});
    const int prec = precision == CPAB_F64 ? PREC_F64 : PREC_F32;
    const int tile_px = likelihood_tile((int64_t)N * H * W * D, ctx->cfg.tile_pts);
    if (register3d_smem_bytes(ctx->t.nC, tile_px, prec) > (size_t)max_smem_optin())
        return fail(ctx, CPAB_UNSUPPORTED, "cell tables and tile scratch exceed shared memory");
    const WsLayout L = ws_layout(N, tiles_of3(H, W, D, kSumChunk));
    if (!workspace || workspace_bytes < L.total)
        return fail(ctx, CPAB_NO_MEMORY, "workspace of %zu bytes needed", L.total);
    Register3dArgs a;
    memset(&a, 0, sizeof(a));
    a.t = ctx->t;
    a.A = signedA;
    a.T = Trels;
    a.src = src;
    a.dst = dst;
    a.warped = warped;
    a.ll = ll;
    char *w = static_cast<char *>(workspace);
    a.partials = reinterpret_cast<double *>(w + L.partials_off);
    a.tickets = reinterpret_cast<unsigned *>(w + L.tickets_off);
    a.counters = reinterpret_cast<unsigned long long *>(counters);
    a.N = N;
    a.H = H;
    a.W = W;
    a.D = D;
    a.tile_px = tile_px;
    a.sigma = sigma;
    a.dt = dt;
    a.nTimeSteps = nTimeSteps;
    a.nStepsODE = nStepsODE;
    a.h_sub = dt / (double)nStepsODE;
    a.cancel = cancel_ptr(ctx);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(a.tickets, 0, (size_t)N * sizeof(unsigned), s);
    if (e != cudaSuccess) return cuda_status(ctx, e, "ticket reset");
    return cuda_status(ctx, launch_register3d_ll(a, prec, ctx->cfg, s), "register3d_ll launch");
}

size_t cpab_landmark_workspace_bytes(const cpab_ctx *ctx, int N, int n_lm)
{
    if (!ctx || N < 0 || n_lm < 1) return 0;
    return ws_layout(N, ((int64_t)n_lm + ctx->cfg.tile_pts - 1) / ctx->cfg.tile_pts).total;
}

int cpab_landmark_ll(cpab_ctx *ctx, const double *signedA, const double *Trels, int N, const double *src,
                     int64_t src_stride, const double *dst, int64_t dst_stride, int n_lm, double sigma, int precision,
                     double dt, int nTimeSteps, int nStepsODE, double *ll, double *transformed, void *workspace,
                     size_t workspace_bytes, uint64_t *counters, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (N < 0 || n_lm < 1) return fail(ctx, CPAB_BAD_SHAPE, "need N >= 0 and n_lm >= 1");
    if (src_stride < 0 || dst_stride < 0) return fail(ctx, CPAB_BAD_SHAPE, "strides must be >= 0");
    if (N == 0) return CPAB_OK;
    if (precision != CPAB_F64 && precision != CPAB_F32)
        return fail(ctx, CPAB_BAD_DTYPE, "precision must be CPAB_F64 or CPAB_F32");
    if (!signedA || !Trels || !src || !dst || !ll) return fail(ctx, CPAB_BAD_ARG, "NULL argument");
    if (!(sigma > 0)) return fail(ctx, CPAB_BAD_ARG, "sigma must be positive");
    if (nTimeSteps < 1 || nStepsODE < 1) return fail(ctx, CPAB_BAD_ARG, "nTimeSteps and nStepsODE must be >= 1");
    if ((long long)nTimeSteps * nStepsODE > 0x7fffffffLL)
        return fail(ctx, CPAB_BAD_ARG, "nTimeSteps * nStepsODE overflows");
    if (!std::isfinite(dt)) return fail(ctx, CPAB_BAD_ARG, "dt is not finite");
    CPAB_CHECK_ALIGN(ctx, {signedA, 8, "signedA"}, {Trels, 8, "Trels"}, {src, 8, "src"}, {dst, 8, "dst"},
                     {ll, 8, "ll"}, {transformed, 8, "transformed"}, {workspace, 8, "workspace"},
                     {counters, 8, "counters"});
    const int prec = precision == CPAB_F64 ? PREC_F64 : PREC_F32;
    if (landmark_smem_bytes(ctx->t, ctx->cfg.tile_pts, prec) > (size_t)max_smem_optin())
        return fail(ctx, CPAB_UNSUPPORTED, "cell tables and tile scratch exceed shared memory");
    const size_t need = cpab_landmark_workspace_bytes(ctx, N, n_lm);
    if (!workspace || workspace_bytes < need) return fail(ctx, CPAB_NO_MEMORY, "workspace of %zu bytes needed", need);
    if (transformed) {
        const size_t tb = (size_t)N * n_lm * ctx->t.dim * 8;
        if (overlaps(transformed, tb, src, (size_t)((N - 1) * src_stride + n_lm) * ctx->t.dim * 8) ||
            overlaps(transformed, tb, dst, (size_t)((N - 1) * dst_stride + n_lm) * ctx->t.dim * 8))
            return fail(ctx, CPAB_ALIAS, "transformed overlaps src or dst");
    }
    const WsLayout L = ws_layout(N, ((int64_t)n_lm + ctx->cfg.tile_pts - 1) / ctx->cfg.tile_pts);
    LandmarkArgs a;
    memset(&a, 0, sizeof(a));
    a.t = ctx->t;
    a.A = signedA;
    a.T = Trels;
    a.src = src;
    a.dst = dst;
    a.src_stride = src_stride;
    a.dst_stride = dst_stride;
    a.transformed = transformed;
    a.ll = ll;
    char *w = static_cast<char *>(workspace);
    a.partials = reinterpret_cast<double *>(w + L.partials_off);
    a.tickets = reinterpret_cast<unsigned *>(w + L.tickets_off);
    a.counters = reinterpret_cast<unsigned long long *>(counters);
    a.N = N;
    a.n_lm = n_lm;
    a.tile_pts = ctx->cfg.tile_pts;
    a.sigma = sigma;
    a.dt = dt;
    a.nTimeSteps = nTimeSteps;
    a.nStepsODE = nStepsODE;
    a.h_sub = dt / (double)nStepsODE;
    a.clamp = ctx->clamp;
    a.clamp_lo = ctx->clamp_lo;
    a.clamp_hi = ctx->clamp_hi;
    a.cancel = cancel_ptr(ctx);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(a.tickets, 0, (size_t)N * sizeof(unsigned), s);
    if (e != cudaSuccess) return cuda_status(ctx, e, "ticket reset");
    return cuda_status(ctx, launch_landmark_ll(a, prec, ctx->cfg, s), "landmark_ll launch");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched Metropolis-Hastings steps (cpab/cpaNd/inference/Metropolis.py:41-85).
#include "cpab_mcmc.h"

namespace {

int check_mcmc(cpab_ctx *ctx, int C, int d, const void *theta, const void *theta_prop, const void *step)
{
    if (C < 0 || d < 1) return fail(ctx, CPAB_BAD_SHAPE, "need C >= 0 chains and d >= 1");
    if (C > 0 && (!theta || !theta_prop || !step)) return fail(ctx, CPAB_BAD_ARG, "theta/theta_prop/step is NULL");
    return CPAB_OK;
}

}  // namespace

extern "C" {

int cpab_mcmc_propose(cpab_ctx *ctx, int C, int d, const double *theta, const double *prop_std, double scale,
                      uint64_t seed, const int64_t *step, double *theta_prop, void *stream)
{
    int st = check_mcmc(ctx, C, d, theta, theta_prop, step);
    if (st != CPAB_OK) return st;
    if (C == 0) return CPAB_OK;
    if (!prop_std) return fail(ctx, CPAB_BAD_ARG, "prop_std is NULL");
    CPAB_CHECK_ALIGN(ctx, {theta, 8, "theta"}, {prop_std, 8, "prop_std"}, {step, 8, "step"},
                     {theta_prop, 8, "theta_prop"});
    if (!std::isfinite(scale)) return fail(ctx, CPAB_BAD_ARG, "scale is not finite");
    McmcArgs a;
    memset(&a, 0, sizeof(a));
    a.C = C;
    a.d = d;
    a.theta = const_cast<double *>(theta);
    a.theta_prop = theta_prop;
    a.prop_std = prop_std;
    a.scale = scale;
    a.seed = seed;
    a.step = const_cast<int64_t *>(step);
    return cuda_status(ctx, launch_mcmc_propose(a, (cudaStream_t)stream), "mcmc_propose launch");
}

int cpab_mcmc_propose_local(cpab_ctx *ctx, int C, int d, const double *theta, int nV, const double *E,
                            const double *G, const int32_t *bdry, double s, uint64_t seed, const int64_t *step,
                            double *theta_prop, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    int st = check_mcmc(ctx, C, d, theta, theta_prop, step);
    if (st != CPAB_OK) return st;
    if (C == 0) return CPAB_OK;
    if (nV < 1) return fail(ctx, CPAB_BAD_SHAPE, "nV < 1");
    if (!E || !G || !bdry) return fail(ctx, CPAB_BAD_ARG, "E/G/bdry is NULL");
    if (!std::isfinite(s)) return fail(ctx, CPAB_BAD_ARG, "s is not finite");
    if ((int64_t)C * 32 > 0x7fffffffLL) return fail(ctx, CPAB_BAD_SHAPE, "too many chains");
    CPAB_CHECK_ALIGN(ctx, {theta, 8, "theta"}, {E, 8, "E"}, {G, 8, "G"}, {bdry, 4, "bdry"}, {step, 8, "step"},
                     {theta_prop, 8, "theta_prop"});
    if (overlaps(theta, (size_t)C * d * 8, theta_prop, (size_t)C * d * 8))
        return fail(ctx, CPAB_ALIAS, "theta and theta_prop overlap");
    LocalProposalArgs a;
    memset(&a, 0, sizeof(a));
    a.C = C;
    a.d = d;
    a.dim = ctx->t.dim;
    a.nV = nV;
    a.theta = theta;
    a.theta_prop = theta_prop;
    a.E = E;
    a.G = G;
    a.bdry = bdry;
    a.s = s;
    a.seed = seed;
    a.step = step;
    return cuda_status(ctx, launch_mcmc_propose_local(a, (cudaStream_t)stream), "mcmc_propose_local launch");
}

int cpab_mcmc_accept(cpab_ctx *ctx, int C, int d, double *theta, const double *theta_prop, double *ll,
                     const double *ll_prop, double inv_npts, const double *prior_prec, double wlp, double *lp,
                     int rule, uint64_t seed, int64_t *step, int64_t *n_accepted, void *stream)
{
    int st = check_mcmc(ctx, C, d, theta, theta_prop, step);
    if (st != CPAB_OK) return st;
    if (rule != 0 && rule != 1) return fail(ctx, CPAB_BAD_ARG, "rule must be 0 (reference) or 1 (textbook)");
    if (prior_prec && !lp) return fail(ctx, CPAB_BAD_ARG, "lp is NULL (needed with prior_prec)");
    if (C > 0) {
        if (!ll || !ll_prop) return fail(ctx, CPAB_BAD_ARG, "ll/ll_prop is NULL");
        CPAB_CHECK_ALIGN(ctx, {theta, 8, "theta"}, {theta_prop, 8, "theta_prop"}, {ll, 8, "ll"},
                         {ll_prop, 8, "ll_prop"}, {prior_prec, 8, "prior_prec"}, {lp, 8, "lp"}, {step, 8, "step"},
                         {n_accepted, 8, "n_accepted"});
        McmcArgs a;
        memset(&a, 0, sizeof(a));
        a.C = C;
        a.d = d;
        a.theta = theta;
        a.theta_prop = const_cast<double *>(theta_prop);
        a.ll = ll;
        a.ll_prop = ll_prop;
        a.inv_npts = inv_npts;
        a.prior_prec = prior_prec;
        a.lp = lp;
        a.wlp = wlp;
        a.rule = rule;
        a.seed = seed;
        a.step = step;
        a.n_accepted = n_accepted;
        cudaError_t e = launch_mcmc_accept(a, (cudaStream_t)stream);
        if (e != cudaSuccess) return cuda_status(ctx, e, "mcmc_accept launch");
    }
    return cuda_status(ctx, step ? launch_mcmc_advance(step, (cudaStream_t)stream) : cudaSuccess,
                       "mcmc_advance launch");
}

// Scratch of cpab_mcmc_run: theta_prop [C, d], signed A and Trel [C, D],
// ll_prop [C], then the registration likelihood's own scratch.
struct McmcRunLayout {
    size_t theta_prop, sA, Tr, ll_prop, reg, total, reg_bytes;
};

static McmcRunLayout mcmc_run_layout(const cpab_ctx *ctx, int C, int d, int H, int W)
{
    McmcRunLayout L;
    const size_t D = (size_t)ctx->t.nC * cell_len(ctx);
    L.theta_prop = 0;
    L.sA = L.theta_prop + align256((size_t)C * d * sizeof(double));
    L.Tr = L.sA + align256((size_t)C * D * sizeof(double));
    L.ll_prop = L.Tr + align256((size_t)C * D * sizeof(double));
    L.reg = L.ll_prop + align256((size_t)C * sizeof(double));
    L.reg_bytes = cpab_register_workspace_bytes(ctx, C, H, W);
    L.total = L.reg + align256(L.reg_bytes);
    return L;
}

size_t cpab_mcmc_run_workspace_bytes(const cpab_ctx *ctx, int C, int d, int H, int W)
{
    if (!ctx || C < 0 || d < 1 || H < 1 || W < 1) return 0;
    return mcmc_run_layout(ctx, C, d, H, W).total;
}

int cpab_mcmc_run(cpab_ctx *ctx, const double *B, int d, int C, double *theta, const double *prop_std, double scale,
                  const float *src, const float *dst, int H, int W, double sigma, int precision, double dt,
                  int nTimeSteps, int nStepsODE, double inv_npts, int rule, uint64_t seed, int64_t *step,
                  int n_steps, double *ll, int64_t *n_accepted, void *workspace, size_t workspace_bytes,
                  void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (ctx->t.dim != 2) return fail(ctx, CPAB_UNSUPPORTED, "the registration chains are built for 2D spaces");
    if (C < 0 || d < 1 || n_steps < 0) return fail(ctx, CPAB_BAD_SHAPE, "need C >= 0, d >= 1, n_steps >= 0");
    if (C == 0) return CPAB_OK;
    if (!B || !theta || !prop_std || !src || !dst || !step || !ll)
        return fail(ctx, CPAB_BAD_ARG, "B/theta/prop_std/src/dst/step/ll is NULL");
    const McmcRunLayout L = mcmc_run_layout(ctx, C, d, H, W);
    if (!workspace || workspace_bytes < L.total)
        return fail(ctx, CPAB_NO_MEMORY, "workspace of %zu bytes needed", L.total);
    CPAB_CHECK_ALIGN(ctx, {workspace, 256, "workspace"});
    char *w = static_cast<char *>(workspace);
    double *theta_prop = reinterpret_cast<double *>(w + L.theta_prop);
    double *sA = reinterpret_cast<double *>(w + L.sA);
    double *Tr = reinterpret_cast<double *>(w + L.Tr);
    double *ll_prop = reinterpret_cast<double *>(w + L.ll_prop);
    void *reg = w + L.reg;
    // the likelihood of the current state, then n_steps Metropolis steps
    int st = cpab_theta_to_trels(ctx, B, d, theta, C, dt, -1, nullptr, sA, Tr, stream);
    if (st == CPAB_OK)
        st = cpab_register_ll(ctx, sA, Tr, C, src, dst, H, W, sigma, precision, dt, nTimeSteps, nStepsODE, ll,
                              nullptr, reg, L.reg_bytes, nullptr, stream);
    for (int k = 0; k < n_steps && st == CPAB_OK; ++k) {
        st = cpab_mcmc_propose(ctx, C, d, theta, prop_std, scale, seed, step, theta_prop, stream);
        if (st == CPAB_OK) st = cpab_theta_to_trels(ctx, B, d, theta_prop, C, dt, -1, nullptr, sA, Tr, stream);
        if (st == CPAB_OK)
            st = cpab_register_ll(ctx, sA, Tr, C, src, dst, H, W, sigma, precision, dt, nTimeSteps, nStepsODE,
                                  ll_prop, nullptr, reg, L.reg_bytes, nullptr, stream);
        if (st == CPAB_OK)
            st = cpab_mcmc_accept(ctx, C, d, theta, theta_prop, ll, ll_prop, inv_npts, nullptr, 0.0, nullptr, rule,
                                  seed, step, n_accepted, stream);
    }
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint gradient of the midpoint scheme (cpab/gpu/calc_2Dto2D.cu:202-319,
// 448-491 computes the same derivative forward; its binding is commented out
// in cpab/gpu/Calcs.py:196).
#include "cpab_grad.h"

extern "C" {

size_t cpab_grad_workspace_bytes(const cpab_ctx *ctx, int N, int64_t n_per_inst, int nTimeSteps, int ck)
{
    if (!ctx || N < 0 || n_per_inst < 0 || nTimeSteps < 1 || ck < 1) return 0;
    const int64_t nck = (nTimeSteps + ck - 1) / ck;
    return align256((size_t)nck * (size_t)N * (size_t)n_per_inst * ctx->t.dim * sizeof(double));
}

size_t cpab_grad_ref_workspace_bytes(const cpab_ctx *ctx, int N, int64_t n_per_inst, int nTimeSteps, int ck)
{
    if (!ctx || N < 0 || n_per_inst < 0 || nTimeSteps < 1 || ck < 1) return 0;
    // checkpoints (FP32: hi and lo per coordinate, the same bytes), then dLoss/dTrels and dLoss/d(sub-step map)
    return cpab_grad_workspace_bytes(ctx, N, n_per_inst, nTimeSteps, ck) +
           2 * align256((size_t)N * ctx->t.nC * cell_len(ctx) * sizeof(double));
}

}  // extern "C"

// Shared body of cpab_grad_theta (ref == false: midpoint scheme, FP64) and
// cpab_grad_theta_ref (reference scheme, needs Trels; FP64 or FP32 points).
static int grad_impl(cpab_ctx *ctx, const double *B, int d, const double *signedA, const double *Trels, bool ref,
                     int N, const void *pts, int64_t n_per_inst, const void *grad_out, int precision, double dt,
                     int nTimeSteps, int nStepsODE, int sign, int ck, void *out, void *grad_pts, double *gA,
                     double *dtheta, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!ctx) return fail(nullptr, CPAB_BAD_ARG, "ctx is NULL");
    if (N < 0 || n_per_inst < 0) return fail(ctx, CPAB_BAD_SHAPE, "N and n_per_inst must be >= 0");
    if (N > 65535) return fail(ctx, CPAB_BAD_SHAPE, "at most 65535 instances per call (got %d)", N);
    if (N == 0) return CPAB_OK;
    if (!signedA || !gA) return fail(ctx, CPAB_BAD_ARG, "signedA/gA is NULL");
    if (ref && !Trels) return fail(ctx, CPAB_BAD_ARG, "Trels is NULL");
    if (dtheta && (!B || d < 1)) return fail(ctx, CPAB_BAD_ARG, "dtheta needs the basis B and d >= 1");
    if (n_per_inst > 0 && (!pts || !grad_out)) return fail(ctx, CPAB_BAD_ARG, "pts/grad_out is NULL");
    if (nTimeSteps < 1 || nStepsODE < 1) return fail(ctx, CPAB_BAD_ARG, "nTimeSteps and nStepsODE must be >= 1");
    if (nStepsODE > 256) return fail(ctx, CPAB_UNSUPPORTED, "the adjoint replays at most 256 sub-steps per step");
    if (ck < 1) return fail(ctx, CPAB_BAD_ARG, "checkpoint stride must be >= 1");
    if (sign != 1 && sign != -1) return fail(ctx, CPAB_BAD_ARG, "sign must be +1 or -1");
    if (!std::isfinite(dt)) return fail(ctx, CPAB_BAD_ARG, "dt is not finite");
    if (precision != CPAB_F64 && precision != CPAB_F32)
        return fail(ctx, CPAB_BAD_DTYPE, "precision must be CPAB_F64 or CPAB_F32");
    if (!ref && precision != CPAB_F64) return fail(ctx, CPAB_UNSUPPORTED, "the midpoint-scheme adjoint is FP64");
    const unsigned pa = precision == CPAB_F64 ? 8u : 4u;
    CPAB_CHECK_ALIGN(ctx, {B, 8, "B"}, {signedA, 8, "signedA"}, {Trels, 8, "Trels"}, {pts, pa, "pts"},
                     {grad_out, pa, "grad_out"}, {out, pa, "out"}, {grad_pts, pa, "grad_pts"}, {gA, 8, "gA"},
                     {dtheta, 8, "dtheta"}, {workspace, 8, "workspace"});
    // tables (reference scheme: the closed-form steps too) in shared memory
    if ((size_t)2 * ctx->t.nC * cell_len(ctx) * 8 > (size_t)max_smem_optin())
        return fail(ctx, CPAB_UNSUPPORTED, "cell tables exceed shared memory");
    const size_t ck_bytes = cpab_grad_workspace_bytes(ctx, N, n_per_inst, nTimeSteps, ck);
    const size_t need = ref ? cpab_grad_ref_workspace_bytes(ctx, N, n_per_inst, nTimeSteps, ck) : ck_bytes;
    if (n_per_inst > 0 && (!workspace || workspace_bytes < need))
        return fail(ctx, CPAB_NO_MEMORY, "workspace of %zu bytes needed", need);
    cudaStream_t s = (cudaStream_t)stream;
    const int DA = ctx->t.nC * cell_len(ctx);
    cudaError_t e = cudaMemsetAsync(gA, 0, (size_t)N * DA * sizeof(double), s);
    if (e != cudaSuccess) return cuda_status(ctx, e, "gA reset");
    if (n_per_inst > 0) {
        GradArgs a;
        memset(&a, 0, sizeof(a));
        a.t = ctx->t;
        a.A = signedA;
        a.T = Trels;
        a.pts = static_cast<const double *>(pts);  // float data when precision is CPAB_F32
        a.grad_out = static_cast<const double *>(grad_out);
        a.out = static_cast<double *>(out);
        a.grad_in = static_cast<double *>(grad_pts);
        a.gA = gA;
        a.ckpt = static_cast<double *>(workspace);
        a.N = N;
        a.n_per_inst = n_per_inst;
        a.dt = dt;
        a.nTimeSteps = nTimeSteps;
        a.nStepsODE = nStepsODE;
        a.ck = ck;
        a.h_sub = dt / (double)nStepsODE;
        if (ref) {
            const size_t sum_bytes = align256((size_t)N * DA * sizeof(double));
            a.gT = reinterpret_cast<double *>(static_cast<char *>(workspace) + ck_bytes);
            a.gS = reinterpret_cast<double *>(static_cast<char *>(workspace) + ck_bytes + sum_bytes);
            e = cudaMemsetAsync(a.gT, 0, 2 * sum_bytes, s);
            if (e != cudaSuccess) return cuda_status(ctx, e, "gradient sums reset");
            e = precision == CPAB_F64 ? launch_grad_ref(a, s) : launch_grad_ref_f32(a, s);
        } else {
            e = launch_grad_simple(a, s);
        }
        if (e != cudaSuccess) return cuda_status(ctx, e, "grad launch");
    }
    if (dtheta) {
        e = launch_bt_times(B, gA, dtheta, DA, d, N, (double)sign, s);
        if (e != cudaSuccess) return cuda_status(ctx, e, "B^T launch");
    }
    return CPAB_OK;
}

extern "C" {

int cpab_grad_theta(cpab_ctx *ctx, const double *B, int d, const double *signedA, int N, const double *pts,
                    int64_t n_per_inst, const double *grad_out, double dt, int nTimeSteps, int nStepsODE, int sign,
                    int ck, double *out, double *grad_pts, double *gA, double *dtheta, void *workspace,
                    size_t workspace_bytes, void *stream)
{
    return grad_impl(ctx, B, d, signedA, nullptr, false, N, pts, n_per_inst, grad_out, CPAB_F64, dt, nTimeSteps,
                     nStepsODE, sign, ck, out, grad_pts, gA, dtheta, workspace, workspace_bytes, stream);
}

int cpab_grad_theta_ref(cpab_ctx *ctx, const double *B, int d, const double *signedA, const double *Trels, int N,
                        const void *pts, int64_t n_per_inst, const void *grad_out, int precision, double dt,
                        int nTimeSteps, int nStepsODE, int sign, int ck, void *out, void *grad_pts, double *gA,
                        double *dtheta, void *workspace, size_t workspace_bytes, void *stream)
{
    return grad_impl(ctx, B, d, signedA, Trels, true, N, pts, n_per_inst, grad_out, precision, dt, nTimeSteps,
                     nStepsODE, sign, ck, out, grad_pts, gA, dtheta, workspace, workspace_bytes, stream);
}

}  // extern "C"
