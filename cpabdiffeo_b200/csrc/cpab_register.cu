// cpab_register.cu -- bilinear remap and the Gaussian SSD log-likelihood.
//
//   k_remap_ssd     warped = bilinear(src, map) (cv2.remap semantics: x = column,
//                   y = row, integer coordinates at pixel centres, taps outside
//                   the image read 0 -- cpab/cpa2d/TransformWrapper.py:286-317),
//                   and optionally ll = sum -0.5 (warped - dst)^2 / sigma^2
//                   (cpab/cpa2d/model/transformations/register/gpu/gaussian.py:15-34,
//                   _ScaleDependentLogLikelihoodGeneral.py:108-131) for N images
//                   in one streaming pass.
//   k_register_ll   the registration likelihood of
//                   _ScaleDependentLogLikelihoodGaussian.calc_ll (:34-109) fused:
//                   every pixel centre of the image is integrated with the
//                   instance's tables (pass the inverse, sign -1, tables to get
//                   calc_T_inv), sampled from src and compared with dst, without
//                   writing the map.
//
// Sums are deterministic.  k_remap_ssd: each tile of pixels reduces in a
// fixed order (lanes, then warps) and writes its partial; a second launch
// adds each image's partials in index order.  k_register_ll: fixed 256-pixel
// chunks (cpab_reduce.cuh finish_tile_chunks), added per image in index
// order by the last tile to finish, so the sum does not depend on the tile
// size either.  A result is therefore the same alone and inside any batch.
#include <cmath>

#include <math_constants.h>

#include "cpab_bulk.cuh"
#include "cpab_integrate.cuh"
#include "cpab_launch.h"
#include "cpab_reduce.cuh"
#include "cpab_register.h"

namespace cpab {

// Bilinear sample of a float image at pixel coordinates (px, py), zero
// outside (cv2 conventions).  floor and fraction are taken in double -- floor
// by adding 1.5 * 2^52 with rounding toward -inf, which leaves floor(px) as an
// integer in the low word, so no conversion instruction is needed.  The taps
// are combined in double for double maps / the FP64 likelihood, and in float
// (weights rounded to float, error <= 3 ulp of the value) for float maps /
// the FP32 likelihood.
struct Taps {
    float v[4];      // (r0, c0), (r0, c0 + 1), (r0 + 1, c0), (r0 + 1, c0 + 1)
    double fx, fy;
    bool in;
};

__device__ __forceinline__ void taps_issue(const float *img, int H, int W, double px, double py, Taps &t)
{
    constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
    const double sx = __dadd_rd(px, kRound), sy = __dadd_rd(py, kRound);
    const double fx0 = sx - kRound, fy0 = sy - kRound;  // floor(px), floor(py) for |p| < 2^51
    t.in = fx0 > -2.0 && fx0 < (double)W + 1.0 && fy0 > -2.0 && fy0 < (double)H + 1.0;  // false for NaN
    t.fx = px - fx0;
    t.fy = py - fy0;
    const int c0 = t.in ? __double2loint(sx) : -2, r0 = t.in ? __double2loint(sy) : -2;
    if (c0 >= 0 && c0 + 1 < W && r0 >= 0 && r0 + 1 < H) {
        // the whole 2x2 footprint is inside (the common case): four unconditional loads
        const float *q = img + (r0 * W + c0);
        t.v[0] = __ldg(q);
        t.v[1] = __ldg(q + 1);
        t.v[2] = __ldg(q + W);
        t.v[3] = __ldg(q + W + 1);
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int r = r0 + (k >> 1), c = c0 + (k & 1);
            t.v[k] = (r >= 0 && r < H && c >= 0 && c < W) ? __ldg(img + (r * W + c)) : 0.0f;
        }
    }
}

template <typename Real>
__device__ __forceinline__ Real taps_combine(const Taps &t);

template <>
__device__ __forceinline__ double taps_combine<double>(const Taps &t)
{
    if (!t.in) return 0.0;
    const double top = (1 - t.fx) * (double)t.v[0] + t.fx * (double)t.v[1];
    const double bot = (1 - t.fx) * (double)t.v[2] + t.fx * (double)t.v[3];
    return (1 - t.fy) * top + t.fy * bot;
}

template <>
__device__ __forceinline__ float taps_combine<float>(const Taps &t)
{
    if (!t.in) return 0.0f;
    const float wx = (float)t.fx, wy = (float)t.fy;
    const float top = fmaf(wx, t.v[1] - t.v[0], t.v[0]);
    const float bot = fmaf(wx, t.v[3] - t.v[2], t.v[2]);
    return fmaf(wy, bot - top, top);
}

template <typename Real>
__device__ __forceinline__ Real bilinear(const float *img, int H, int W, double px, double py)
{
    Taps t;
    taps_issue(img, H, W, px, py, t);
    return taps_combine<Real>(t);
}

// Float coordinates for float maps whose pixel mapping is exact in float: px
// = fma(x, sx, ox) with sx a power of two and ox 0 or -0.5 is exact except
// for points left of the image, where it is off by at most ~1e-7 pixel (the
// host sets RemapArgs::fcoord only then).  floor by adding 1.5 * 2^23 with
// rounding toward -inf; taps combined in float as taps_combine<float>.
// Split in issue (the four loads) and combine so that a thread can keep the
// taps of several pixels in flight.
__device__ __forceinline__ float2 neg2f(float2 a) { return make_float2(-a.x, -a.y); }

struct TapsF {
    float v[4];
    float wx, wy;
    bool in;
};

__device__ __forceinline__ void tapsf_issue(const float *img, int H, int W, float px, float py, TapsF &t)
{
    // x and y as one pair (sm_100's FADD2; each lane rounds as its scalar twin)
    constexpr float kRound = 12582912.0f;  // 1.5 * 2^23
    const float2 p2 = make_float2(px, py);
    const float2 s2 = __fadd2_rd(p2, make_float2(kRound, kRound));
    const float2 f2 = __fadd2_rn(s2, make_float2(-kRound, -kRound));  // floor(px), floor(py) for |p| < 2^22
    const float sx = s2.x, sy = s2.y, fx0 = f2.x, fy0 = f2.y;
    t.in = fx0 > -2.0f && fx0 < (float)W + 1.0f && fy0 > -2.0f && fy0 < (float)H + 1.0f;  // false for NaN
    const float2 w2 = __fadd2_rn(p2, make_float2(-fx0, -fy0));
    t.wx = w2.x;
    t.wy = w2.y;
    const int c0 = t.in ? __float_as_int(sx) - 0x4B400000 : -2;
    const int r0 = t.in ? __float_as_int(sy) - 0x4B400000 : -2;
    if ((unsigned)c0 < (unsigned)(W - 1) && (unsigned)r0 < (unsigned)(H - 1)) {
        const float *q = img + (r0 * W + c0);
        t.v[0] = __ldg(q);
        t.v[1] = __ldg(q + 1);
        t.v[2] = __ldg(q + W);
        t.v[3] = __ldg(q + W + 1);
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int r = r0 + (k >> 1), c = c0 + (k & 1);
            t.v[k] = (r >= 0 && r < H && c >= 0 && c < W) ? __ldg(img + (r * W + c)) : 0.0f;
        }
    }
}

__device__ __forceinline__ float tapsf_combine(const TapsF &t)
{
    if (!t.in) return 0.0f;
    // top and bottom rows as one pair: fmaf(wx, v1 - v0, v0), fmaf(wx, v3 - v2, v2)
    const float2 lo = make_float2(t.v[0], t.v[2]);
    const float2 tb = __ffma2_rn(make_float2(t.wx, t.wx), __fadd2_rn(make_float2(t.v[1], t.v[3]), neg2f(lo)), lo);
    return fmaf(t.wy, tb.y - tb.x, tb.x);
}

__device__ __forceinline__ float bilinear_f(const float *img, int H, int W, float px, float py)
{
    TapsF t;
    tapsf_issue(img, H, W, px, py, t);
    return tapsf_combine(t);
}

// One remap sample in the map's arithmetic (FCOORD: float coordinates).
template <typename MapT, bool FCOORD>
__device__ __forceinline__ MapT remap_sample(const RemapArgs &a, const float *src, MapT mx, MapT my)
{
    if (FCOORD)
    {
        const float2 p = __ffma2_rn(make_float2((float)mx, (float)my), make_float2((float)a.sx, (float)a.sy),
                                    make_float2((float)a.ox, (float)a.oy));
        return (MapT)bilinear_f(src, a.H, a.W, p.x, p.y);
    }
    return bilinear<MapT>(src, a.H, a.W, (double)mx * a.sx + a.ox, (double)my * a.sy + a.oy);
}

// ------------------------------------------------------------ standalone remap (+ SSD)

// (x, y) of one map entry in shared memory with one 8- or 16-byte load.
__device__ __forceinline__ void load_pair(const float *p, float &x, float &y)
{
    const float2 v = *reinterpret_cast<const float2 *>(p);
    x = v.x;
    y = v.y;
}
__device__ __forceinline__ void load_pair(const double *p, double &x, double &y)
{
    const double2 v = *reinterpret_cast<const double2 *>(p);
    x = v.x;
    y = v.y;
}

// Plain path (any alignment, any image size): one pixel per thread and
// iteration, pixels in increasing order per thread.
template <typename MapT, bool FCOORD>
__global__ void __launch_bounds__(256) k_remap_ssd(RemapArgs a)
{
    const int inst = blockIdx.y;
    const int64_t npx = (int64_t)a.H * a.W;
    const int64_t tile = blockIdx.x;
    const int64_t start = tile * a.tile_px;
    const int n = (int)(min(start + (int64_t)a.tile_px, npx) - start);
    const int64_t off = (int64_t)inst * npx + start;
    const MapT *map = static_cast<const MapT *>(a.map) + 2 * off;
    const float *src = a.src + (int64_t)inst * npx;
    const float *dst = a.dst ? a.dst + off : nullptr;
    float *warped = a.warped ? a.warped + off : nullptr;
    const double k = -0.5 / (a.sigma * a.sigma);
    double acc = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const MapT w = remap_sample<MapT, FCOORD>(a, src, map[2 * j], map[2 * j + 1]);
        if (warped) warped[j] = (float)w;
        if (dst) {
            const double e = (double)w - (double)__ldg(dst + j);
            acc += e * e * k;
        }
    }
    if (dst) store_tile_partial(acc, 0, (int64_t)inst * gridDim.x + tile, a.partials);
}

// Bulk path (16-byte aligned map and dst, H*W a multiple of 4): a persistent
// grid walks the (image, tile) list; while a CTA samples one tile, the map
// and dst of its next tile stream into the other shared-memory stage by
// cp.async.bulk, so the only loads the threads wait on are the source taps.
// Same per-pixel arithmetic and per-thread order as the plain path, hence
// the same results.  A stage whose copy does not complete within the wait
// bound makes that tile's partial (hence its image's ll) NaN and leaves its
// warped tile unwritten; the CTA then issues no further copies, marks its
// remaining tiles NaN without waiting, and before exiting waits once more
// (bounded) for the copies it has in flight -- a copy still outstanding after
// that second bound may land in the CTA's shared memory after it exits.
// One tile of the float-coordinate path: four pixels' taps in flight per
// thread; sums in pixel order.  FAST: a full tile (n a multiple of four
// blocks), SSD on, no warped output -- no per-pixel checks.
constexpr int kRemapInFlight = 4;
template <bool FAST, typename MapT>
__device__ __forceinline__ void remap_tile_f(const RemapArgs &a, const MapT *m, const float *dv, const float *src,
                                             float *warped, int n, double k, double &acc)
{
    constexpr int kB = kRemapInFlight;
    for (int j0 = threadIdx.x; j0 < n; j0 += kB * blockDim.x) {
        TapsF t[kB];
#pragma unroll
        for (int u = 0; u < kB; ++u) {
            const int j = j0 + u * blockDim.x;
            t[u].in = false;
            if (FAST || j < n) {
                MapT mx, my;
                load_pair(m + 2 * j, mx, my);
                const float2 pp = __ffma2_rn(make_float2((float)mx, (float)my), make_float2((float)a.sx, (float)a.sy),
                                             make_float2((float)a.ox, (float)a.oy));
                tapsf_issue(src, a.H, a.W, pp.x, pp.y, t[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < kB; ++u) {
            const int j = j0 + u * blockDim.x;
            if (FAST || j < n) {
                const float w = tapsf_combine(t[u]);
                if (!FAST && warped) warped[j] = w;
                if (FAST || a.dst) {
                    const double e = (double)w - (double)dv[j];
                    acc += e * e * k;
                }
            }
        }
    }
}

// Launch shape, measured on 256 pairs of 256^2 images through float maps
// (same box): 3 CTAs of 256 threads per SM (80 registers) with the fast
// full-tile path 0.092 ms; 4 CTAs (64 registers, spilling) 0.104 ms; 2 CTAs
// 0.107 ms; 6 or 8 pixels in flight per thread instead of 4: 0.109 / 0.115 ms.
template <typename MapT, bool FCOORD>
__global__ void __launch_bounds__(256, 3) k_remap_ssd_bulk(RemapArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ int s_dead;  // a wait of this CTA gave up
    const int TP = a.tile_px;
    // stage s: map at s_map0 + s * 2 TP, dst at s_dst0 + s * TP
    MapT *const s_map0 = reinterpret_cast<MapT *>(smem_raw);
    float *const s_dst0 = reinterpret_cast<float *>(s_map0 + 4 * TP);
    const int64_t npx = (int64_t)a.H * a.W;
    const int tpi = (int)((npx + TP - 1) / TP);
    const int64_t ntiles = (int64_t)tpi * a.N;
    const double k = -0.5 / (a.sigma * a.sigma);
    const MapT *gmap = static_cast<const MapT *>(a.map);
    if (threadIdx.x == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_fence_init();
        s_dead = 0;
    }
    __syncthreads();
    int issued0 = 0, issued1 = 0;  // copies thread 0 issued per stage (one phase each)
    // (image, tile within the image) of the current tile, advanced by the
    // grid stride with one add and one compare instead of a 64-bit division
    // per tile: stride = qG images + rG tiles
    const int64_t qG = (int64_t)gridDim.x / tpi, rG = (int64_t)gridDim.x - qG * tpi;
    auto advance = [&](int64_t &inst, int64_t &tin) {
        tin += rG;
        inst += qG;
        if (tin >= tpi) {
            tin -= tpi;
            ++inst;
        }
    };
    auto issue = [&](int64_t inst, int64_t tin, int stage) {
        if (stage) ++issued1; else ++issued0;
        const int64_t start = tin * TP;
        const int n = (int)min((int64_t)TP, npx - start);
        const int64_t off = inst * npx + start;
        const uint32_t mb = (uint32_t)n * 2u * (uint32_t)sizeof(MapT), db = a.dst ? (uint32_t)n * 4u : 0u;
        mbar_arrive_expect_tx(&s_bar[stage], mb + db);
        bulk_g2s(s_map0 + stage * 2 * TP, gmap + 2 * off, mb, &s_bar[stage]);
        if (db) bulk_g2s(s_dst0 + stage * TP, a.dst + off, db, &s_bar[stage]);
    };
    int64_t inst = (int64_t)blockIdx.x / tpi, tin = (int64_t)blockIdx.x - inst * tpi;
    if (threadIdx.x == 0 && (int64_t)blockIdx.x < ntiles) issue(inst, tin, 0);
    int it = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int stage = it & 1;
        const uint32_t parity = (uint32_t)(it >> 1) & 1u;
        int64_t inst_n = inst, tin_n = tin;
        advance(inst_n, tin_n);
        // s_dead was last written before the previous tile's closing barrier
        const bool dead = s_dead != 0;
        // the other stage was released by the previous iteration's closing barrier
        if (threadIdx.x == 0 && !dead && tile + gridDim.x < ntiles) issue(inst_n, tin_n, stage ^ 1);
        const bool ok = !dead && mbar_wait(&s_bar[stage], parity);
        if (!ok && !dead) s_dead = 1;
        const int64_t start = tin * TP;
        const int n = (int)min((int64_t)TP, npx - start);
        const int64_t off = inst * npx + start;
        const float *src = a.src + inst * npx;
        float *warped = a.warped ? a.warped + off : nullptr;
        double acc = 0.0;
        if (ok && FCOORD) {
            const MapT *m = s_map0 + stage * 2 * TP;
            const float *dv = s_dst0 + stage * TP;
            // the common case -- a full tile, SSD, no warped output -- without
            // per-pixel bounds and option checks
            if (a.dst && !warped && n % (kRemapInFlight * (int)blockDim.x) == 0)
                remap_tile_f<true>(a, m, dv, src, nullptr, n, k, acc);
            else
                remap_tile_f<false>(a, m, dv, src, warped, n, k, acc);
        } else if (ok) {
            const MapT *m = s_map0 + stage * 2 * TP;
            const float *dv = s_dst0 + stage * TP;
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                MapT mx, my;
                load_pair(m + 2 * j, mx, my);
                const MapT w = remap_sample<MapT, FCOORD>(a, src, mx, my);
                if (warped) warped[j] = (float)w;
                if (a.dst) {
                    const double e = (double)w - (double)dv[j];
                    acc += e * e * k;
                }
            }
        } else {
            acc = CUDART_NAN;
        }
        if (a.dst)
            store_tile_partial(acc, it & 1, tile, a.partials);
        else
            __syncthreads();
        inst = inst_n;
        tin = tin_n;
    }
    // Without a give-up every copy this CTA issued was waited for above (the
    // last issue targets its last tile).  After one, wait (bounded) for the
    // last phase issued to each stage before the shared memory is released.
    if (threadIdx.x == 0 && s_dead) {
        if (issued0) mbar_wait(&s_bar[0], (uint32_t)(issued0 - 1) & 1u);
        if (issued1) mbar_wait(&s_bar[1], (uint32_t)(issued1 - 1) & 1u);
    }
}

template <typename MapT, bool FCOORD>
static cudaError_t launch_remap_bulk(const RemapArgs &a, cudaStream_t s)
{
    auto kern = k_remap_ssd_bulk<MapT, FCOORD>;
    const size_t smem = 2 * (size_t)a.tile_px * (2 * sizeof(MapT) + sizeof(float));
    if (smem > kSmemOptInAbove) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    LaunchCfg cfg;
    cfg.block = 256;
    const int64_t npx = (int64_t)a.H * a.W;
    const int64_t ntiles = ((npx + a.tile_px - 1) / a.tile_px) * a.N;
    int64_t grid = persistent_grid(kern, cfg, smem);
    if (grid > ntiles) grid = ntiles;
    kern<<<(unsigned)grid, 256, smem, s>>>(a);
    return cudaGetLastError();
}

// ll[inst] = sum of the instance's tile partials in index order (the same
// order, hence the same value, as the last-tile summation of finish_tile).
static __global__ void k_sum_partials(const double *partials, int tiles_per_inst, int N, double *ll)
{
    const int inst = blockIdx.x * blockDim.x + threadIdx.x;
    if (inst >= N) return;
    const double *p = partials + (int64_t)inst * tiles_per_inst;
    double tot = 0.0;
    for (int k = 0; k < tiles_per_inst; ++k) tot += p[k];
    ll[inst] = tot;
}

static bool pow2(double v)
{
    int e = 0;
    return v > 0 && std::frexp(v, &e) == 0.5;
}

cudaError_t launch_remap_ssd(const RemapArgs &a, int map_prec, cudaStream_t s)
{
    const int64_t npx = (int64_t)a.H * a.W;
    // float coordinates are exact for power-of-two scales with offsets 0 or -0.5
    const bool fcoord = map_prec == PREC_F32 && pow2(a.sx) && pow2(a.sy) && a.sx <= 4194304.0 &&
                        a.sy <= 4194304.0 && (a.ox == 0.0 || a.ox == -0.5) && (a.oy == 0.0 || a.oy == -0.5) &&
                        a.W < (1 << 22) && a.H < (1 << 22);
    // bulk copies need 16-byte aligned sources and sizes: aligned bases and 4 | H*W
    // (tiles then start at multiples of 4 pixels and hold a multiple of 4)
    const bool bulk = (npx % 4 == 0) && (a.tile_px % 4 == 0) &&
                      (reinterpret_cast<uintptr_t>(a.map) % 16 == 0) &&
                      (!a.dst || reinterpret_cast<uintptr_t>(a.dst) % 16 == 0);
    cudaError_t e;
    if (bulk) {
        if (map_prec == PREC_F64) e = launch_remap_bulk<double, false>(a, s);
        else e = fcoord ? launch_remap_bulk<float, true>(a, s) : launch_remap_bulk<float, false>(a, s);
    } else {
        dim3 grid((unsigned)((npx + a.tile_px - 1) / a.tile_px), (unsigned)a.N);
        if (map_prec == PREC_F64) k_remap_ssd<double, false><<<grid, 256, 0, s>>>(a);
        else if (fcoord) k_remap_ssd<float, true><<<grid, 256, 0, s>>>(a);
        else k_remap_ssd<float, false><<<grid, 256, 0, s>>>(a);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess || !a.dst) return e;
    // per-image sums of the tile partials, in tile order
    const int tpi = (int)((npx + a.tile_px - 1) / a.tile_px);
    k_sum_partials<<<(a.N + 127) / 128, 128, 0, s>>>(a.partials, tpi, a.N, a.ll);
    return cudaGetLastError();
}

// ------------------------------------------------------------ fused registration likelihood

// Start and end points of the current tile's pixels live in shared memory,
// one double2 slot per pixel.  A convergent pass writes the pixel centres
// ((col+0.5)/W, (row+0.5)/H); the lane loop takes a point's start from its
// slot and writes its end point back; a second convergent pass samples src
// at the end points, compares with dst and sums the terms, thread t taking
// pixels t, t + blockDim, ... of the tile (a fixed order, so results do not
// depend on which warp integrated which pixel).  The pixel-index arithmetic
// and the sampling stay out of the lane loop, whose register count sets the
// CTAs per SM, and each warp samples 32 consecutive pixels together.
struct SlotSrc2 {
    const double2 *slot;
    int64_t tile_start;
    template <typename Real>
    __device__ __forceinline__ void load(int64_t i, PState<2, Real> &st) const
    {
        const double2 v = slot[i - tile_start];
        const double p[2] = {v.x, v.y};
        st.set(p);
    }
};

struct SlotSnk2 {
    double2 *slot;
    int64_t tile_start;
    template <typename Real>
    __device__ __forceinline__ void put(int64_t i, const PState<2, Real> &st)
    {
        double p[2];
        st.get(p);
        slot[i - tile_start] = make_double2(p[0], p[1]);
    }
};

// CPAB_REGISTER_MIN_BLOCKS: resident CTAs of 256 threads the register
// allocation must allow per SM (unset: the compiler's own choice).
#ifdef CPAB_REGISTER_MIN_BLOCKS
#define CPAB_REGISTER_BOUNDS __launch_bounds__(256, CPAB_REGISTER_MIN_BLOCKS)
#else
#define CPAB_REGISTER_BOUNDS __launch_bounds__(256)
#endif
template <int TESS, typename Real>
__global__ void CPAB_REGISTER_BOUNDS k_register_ll(RegisterArgs a)
{
    constexpr int DIM = 2, NE = 6;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real *sA = reinterpret_cast<Real *>(smem_raw);
    Real *sT = sA + a.t.nC * NE;
    // the tile's point slots, after the tables (48 or 96 bytes per cell: 16-byte aligned), then the
    // 32-point group sums of the likelihood
    double2 *s_pos = reinterpret_cast<double2 *>(sA + (1 + TableLayout<Real>::kTParts) * a.t.nC * NE);
    double *s_grp = reinterpret_cast<double *>(s_pos + a.tile_px);
    __shared__ unsigned long long s_claim;
    const int tab = a.t.nC * NE;
    const Real h = (Real)(a.dt / (double)a.nStepsODE);
    const int64_t npx = (int64_t)a.H * a.W;
    const int64_t tpi = (npx + a.tile_px - 1) / a.tile_px;
    const int64_t ntiles = tpi * a.N;
    const int cpi = (int)((npx + kSumChunk - 1) / kSumChunk);  // chunk partials per image
    unsigned long long c_fast = 0, c_fb = 0, c_sub = 0, c_pts = 0;
    int loaded = -1;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if ((((tile - blockIdx.x) / gridDim.x) & 7) == 0 && cta_cancelled(a.cancel, a.counters)) break;
        const int inst = (int)(tile / tpi);
        const int64_t kt = tile - (int64_t)inst * tpi;
        const int64_t base = (int64_t)inst * npx;
        const int64_t j0 = kt * a.tile_px;  // first pixel of the tile in its image (a multiple of kSumChunk)
        const int64_t start = base + j0;
        const int n = (int)(min(start + (int64_t)a.tile_px, base + npx) - start);
        if (inst != loaded) {
            __syncthreads();
            stage_tables<DIM, Real>(a.A + (size_t)inst * tab, a.T + (size_t)inst * tab, a.t.nC, true,
                                    a.h_sub, sA, sT);
            loaded = inst;
        }
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int64_t q = j0 + j, r = q / a.W, c = q - r * a.W;
            s_pos[j] = make_double2(((double)c + 0.5) / (double)a.W, ((double)r + 0.5) / (double)a.H);
        }
        if (threadIdx.x == 0) s_claim = 0ull;
        __syncthreads();
        // all warps share the tile through the claim counter
        const SlotSrc2 src{s_pos, start};
        SlotSnk2 snk{s_pos, start};
        integrate_range<DIM, TESS, Real, SCHEME_REF>(a.t, a.nTimeSteps, a.nStepsODE, sA, sT, start, start + n, h,
                                                     src, snk, c_fast, c_fb, c_sub, c_pts, nullptr, 0, &s_claim);
        __syncthreads();
        const float *img = a.src + base, *ref = a.dst + base;
        float *warped = a.warped ? a.warped + base : nullptr;
        const double k = -0.5 / (a.sigma * a.sigma);
        // each pixel's term replaces the x of its slot, then the chunk-ordered sum
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double2 p = s_pos[j];
            const Real w = bilinear<Real>(img, a.H, a.W, p.x * a.W - 0.5, p.y * a.H - 0.5);
            if (warped) warped[j0 + j] = (float)w;
            const double e = (double)w - (double)__ldg(ref + j0 + j);
            s_pos[j].x = __dmul_rn(__dmul_rn(e, e), k);
        }
        __syncthreads();
        finish_tile_chunks(n, [&](int j) { return s_pos[j].x; }, s_grp, (int64_t)inst * cpi + j0 / kSumChunk, inst,
                           (int)tpi, cpi, a.partials, a.tickets, a.ll);
    }
    if (a.counters) {
        c_fast = warp_sum_u64(c_fast);
        c_fb = warp_sum_u64(c_fb);
        c_sub = warp_sum_u64(c_sub);
        c_pts = warp_sum_u64(c_pts);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(a.counters + CNT_FAST, c_fast);
            atomicAdd(a.counters + CNT_FALLBACK, c_fb);
            atomicAdd(a.counters + CNT_SUBSTEPS, c_sub);
            atomicAdd(a.counters + CNT_POINTS, c_pts);
        }
    }
}

size_t register_smem_bytes(int nC, int tile_px, int prec)
{
    return (size_t)nC * 6 * (prec == PREC_F64 ? 2 * 8 : 2 * 4) + (size_t)tile_px * sizeof(double2) +
           (size_t)((tile_px + 31) / 32) * sizeof(double);
}

template <int TESS, typename Real>
static cudaError_t launch_register_t(const RegisterArgs &a, const LaunchCfg &cfg, cudaStream_t s)
{
    const size_t smem = register_smem_bytes(a.t.nC, a.tile_px, sizeof(Real) == 8 ? PREC_F64 : PREC_F32);
    auto kern = k_register_ll<TESS, Real>;
    if (smem > kSmemOptInAbove) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int64_t npx = (int64_t)a.H * a.W;
    const int64_t ntiles = ((npx + a.tile_px - 1) / a.tile_px) * a.N;
    int64_t grid = persistent_grid(kern, cfg, smem);
    if (grid > ntiles) grid = ntiles;
    kern<<<(unsigned)grid, cfg.block, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_register_ll(const RegisterArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s)
{
    if (a.t.tess == 1)
        return prec == PREC_F64 ? launch_register_t<1, double>(a, cfg, s) : launch_register_t<1, float>(a, cfg, s);
    return prec == PREC_F64 ? launch_register_t<2, double>(a, cfg, s) : launch_register_t<2, float>(a, cfg, s);
}

}  // namespace cpab
