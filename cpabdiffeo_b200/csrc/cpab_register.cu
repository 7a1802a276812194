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
// Sums are deterministic: each tile of pixels reduces in a fixed order
// (lanes, then warps), writes its partial, and the last tile of an image to
// finish (atomic ticket with fences) adds that image's partials in index
// order.  A result is therefore the same alone and inside any batch.
#include "cpab_integrate.cuh"
#include "cpab_launch.h"
#include "cpab_register.h"

namespace cpab {

// Bilinear sample of a float image at pixel coordinates (px, py), zero outside.
__device__ __forceinline__ double tap(const float *img, int H, int W, int r, int c)
{
    return (r >= 0 && r < H && c >= 0 && c < W) ? (double)__ldg(img + (int64_t)r * W + c) : 0.0;
}

__device__ __forceinline__ double bilinear(const float *img, int H, int W, double px, double py)
{
    double fx0 = floor(px), fy0 = floor(py);
    if (!(fx0 > -2.0 && fx0 < (double)W + 1.0 && fy0 > -2.0 && fy0 < (double)H + 1.0)) return 0.0;
    double fx = px - fx0, fy = py - fy0;
    int c0 = (int)fx0, r0 = (int)fy0;
    double top = (1 - fx) * tap(img, H, W, r0, c0) + fx * tap(img, H, W, r0, c0 + 1);
    double bot = (1 - fx) * tap(img, H, W, r0 + 1, c0) + fx * tap(img, H, W, r0 + 1, c0 + 1);
    return (1 - fy) * top + fy * bot;
}

__device__ __forceinline__ double warp_sum_f64(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    return v;
}

// Reduce `acc` over the CTA (fixed order) and hand the tile's partial to the
// per-image bookkeeping.  All threads of the CTA must call this.
__device__ void finish_tile(double acc, int64_t tile, int inst, int tiles_of_inst, int64_t first_tile_of_inst,
                            double *partials, unsigned *tickets, double *ll_out)
{
    __shared__ double s_w[32];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    acc = warp_sum_f64(acc);
    if (lane == 0) s_w[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += s_w[w];
        partials[tile] = s;
        __threadfence();
        unsigned ticket = atomicAdd(tickets + inst, 1u);
        s_last = (ticket == (unsigned)tiles_of_inst - 1u);
        if (s_last) {
            __threadfence();
            double tot = 0.0;
            for (int k = 0; k < tiles_of_inst; ++k) tot += ((volatile double *)partials)[first_tile_of_inst + k];
            ll_out[inst] = tot;
            tickets[inst] = 0u;  // ready for the next call
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------ standalone remap (+ SSD)

__device__ __forceinline__ void load_pair(const float *p, float &x, float &y)
{
    const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
    x = v.x;
    y = v.y;
}

__device__ __forceinline__ void load_pair(const double *p, double &x, double &y)
{
    const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    x = v.x;
    y = v.y;
}

// Bilinear sampling split in two halves so that a thread can issue the tap
// loads of several pixels before it needs any of them: same arithmetic as
// bilinear().
struct TapSet {
    float v[4];      // (r0, c0), (r0, c0 + 1), (r0 + 1, c0), (r0 + 1, c0 + 1)
    double fx, fy;
    bool inside;
};

__device__ __forceinline__ void taps_issue(const float *img, int H, int W, double px, double py, TapSet &t)
{
    const double fx0 = floor(px), fy0 = floor(py);
    t.inside = fx0 > -2.0 && fx0 < (double)W + 1.0 && fy0 > -2.0 && fy0 < (double)H + 1.0;
    t.fx = px - fx0;
    t.fy = py - fy0;
    const int c0 = t.inside ? (int)fx0 : -2, r0 = t.inside ? (int)fy0 : -2;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = r0 + (k >> 1), c = c0 + (k & 1);
        t.v[k] = (r >= 0 && r < H && c >= 0 && c < W) ? __ldg(img + (int64_t)r * W + c) : 0.0f;
    }
}

__device__ __forceinline__ double taps_combine(const TapSet &t)
{
    if (!t.inside) return 0.0;
    const double top = (1 - t.fx) * (double)t.v[0] + t.fx * (double)t.v[1];
    const double bot = (1 - t.fx) * (double)t.v[2] + t.fx * (double)t.v[3];
    return (1 - t.fy) * top + t.fy * bot;
}

// Each thread handles kRemapBatch pixels per round (stride blockDim.x, so a
// warp's accesses stay coalesced): all map and dst loads of the round are
// issued first, then all tap loads, then the arithmetic -- enough loads in
// flight per SM to stream HBM.  Per-thread sums keep pixel order.
constexpr int kRemapBatch = 4;

template <typename MapT>
__global__ void __launch_bounds__(256, 3) k_remap_ssd(RemapArgs a)
{
    const int inst = blockIdx.y;
    const int64_t npx = (int64_t)a.H * a.W;
    const int64_t tile = blockIdx.x;
    const int64_t start = tile * a.tile_px;
    const int n = (int)(min(start + (int64_t)a.tile_px, npx) - start);   // pixels of this tile
    // tile-relative pointers: the per-pixel indices below are 32-bit
    const int64_t off = (int64_t)inst * npx + start;
    const MapT *map = static_cast<const MapT *>(a.map) + 2 * off;
    const float *src = a.src + (int64_t)inst * npx;
    const float *dst = a.dst ? a.dst + off : nullptr;
    float *warped = a.warped ? a.warped + off : nullptr;
    const double k = -0.5 / (a.sigma * a.sigma);
    double acc = 0.0;
    // one vector load per (x, y) pair when the map is aligned for it (uniform over the launch)
    const bool vec = (reinterpret_cast<uintptr_t>(a.map) & (2 * sizeof(MapT) - 1)) == 0;
    for (int j0 = threadIdx.x; j0 < n; j0 += kRemapBatch * blockDim.x) {
        MapT mx[kRemapBatch], my[kRemapBatch];
        float dv[kRemapBatch];
#pragma unroll
        for (int u = 0; u < kRemapBatch; ++u) {
            const int j = j0 + u * blockDim.x;
            mx[u] = my[u] = 0;
            dv[u] = 0.0f;
            if (j < n) {
                if (vec) {
                    load_pair(map + 2 * j, mx[u], my[u]);
                } else {
                    mx[u] = map[2 * j];
                    my[u] = map[2 * j + 1];
                }
                if (dst) dv[u] = __ldg(dst + j);
            }
        }
        TapSet ts[kRemapBatch];
#pragma unroll
        for (int u = 0; u < kRemapBatch; ++u) {
            if (j0 + u * (int)blockDim.x < n)
                taps_issue(src, a.H, a.W, (double)mx[u] * a.sx + a.ox, (double)my[u] * a.sy + a.oy, ts[u]);
        }
#pragma unroll
        for (int u = 0; u < kRemapBatch; ++u) {
            const int j = j0 + u * blockDim.x;
            if (j < n) {
                const double w = taps_combine(ts[u]);
                if (warped) warped[j] = (float)w;
                if (dst) {
                    const double e = w - (double)dv[u];
                    acc += e * e * k;
                }
            }
        }
    }
    if (dst) {
        const int tpi = (int)gridDim.x;
        finish_tile(acc, (int64_t)inst * tpi + tile, inst, tpi, (int64_t)inst * tpi, a.partials, a.tickets, a.ll);
    }
}

cudaError_t launch_remap_ssd(const RemapArgs &a, int map_prec, cudaStream_t s)
{
    const int64_t npx = (int64_t)a.H * a.W;
    dim3 grid((unsigned)((npx + a.tile_px - 1) / a.tile_px), (unsigned)a.N);
    if (map_prec == PREC_F64) k_remap_ssd<double><<<grid, 256, 0, s>>>(a);
    else k_remap_ssd<float><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ------------------------------------------------------------ fused registration likelihood

// Start points: the pixel centres ((col+0.5)/W, (row+0.5)/H) of instance
// inst's image; the point index within the instance is row-major.
struct PixelSrc {
    int H, W;
    int64_t base;  // first global index of the instance
    template <typename Real>
    __device__ __forceinline__ void load(int64_t i, PState<2, Real> &st) const
    {
        const int64_t j = i - base;
        const int64_t r = j / W, c = j - r * W;
        double p[2];
        p[0] = ((double)c + 0.5) / (double)W;
        p[1] = ((double)r + 0.5) / (double)H;
        st.set(p);
    }
};

// End points: sampled from src and scored against dst; nothing stored
// unless `warped` is given.  Each pixel's term goes to its slot of the
// tile's shared-memory array, so the tile sum can be taken in a fixed order
// whichever warp finished the pixel.
struct SsdSnk {
    const float *src, *dst;
    float *warped;
    int H, W;
    int64_t base, tile_start;
    double k;
    double *term;
    template <typename Real>
    __device__ __forceinline__ void put(int64_t i, const PState<2, Real> &st)
    {
        const int64_t j = i - base;
        double p[2];
        st.get(p);
        double w = bilinear(src, H, W, p[0] * W - 0.5, p[1] * H - 0.5);
        if (warped) warped[j] = (float)w;
        double e = w - (double)__ldg(dst + j);
        term[i - tile_start] = e * e * k;
    }
};

template <int TESS, typename Real>
__global__ void __launch_bounds__(256) k_register_ll(RegisterArgs a)
{
    constexpr int DIM = 2, NE = 6;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real *sA = reinterpret_cast<Real *>(smem_raw);
    Real *sT = sA + a.t.nC * NE;
    // per-pixel terms of the current tile, after the tables (their size is a multiple of 8 bytes)
    double *s_term = reinterpret_cast<double *>(sA + (1 + TableLayout<Real>::kTParts) * a.t.nC * NE);
    __shared__ unsigned long long s_claim;
    const int tab = a.t.nC * NE;
    const Real h = (Real)(a.dt / (double)a.nStepsODE);
    const int64_t npx = (int64_t)a.H * a.W;
    const int64_t tpi = (npx + a.tile_px - 1) / a.tile_px;
    const int64_t ntiles = tpi * a.N;
    unsigned long long c_fast = 0, c_fb = 0, c_sub = 0, c_pts = 0;
    int loaded = -1;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if ((((tile - blockIdx.x) / gridDim.x) & 7) == 0 && cta_cancelled(a.cancel, a.counters)) break;
        const int inst = (int)(tile / tpi);
        const int64_t k = tile - (int64_t)inst * tpi;
        const int64_t base = (int64_t)inst * npx;
        const int64_t start = base + k * a.tile_px;
        const int64_t end = min(start + (int64_t)a.tile_px, base + npx);
        if (inst != loaded) {
            __syncthreads();
            stage_tables<DIM, Real>(a.A + (size_t)inst * tab, a.T + (size_t)inst * tab, a.t.nC, true, sA, sT);
            loaded = inst;
            __syncthreads();
        }
        PixelSrc src{a.H, a.W, base};
        SsdSnk snk{a.src + base, a.dst + base, a.warped ? a.warped + base : nullptr, a.H, a.W, base, start,
                   -0.5 / (a.sigma * a.sigma), s_term};
        if (threadIdx.x == 0) s_claim = 0ull;
        __syncthreads();
        // all warps share the tile through the claim counter
        integrate_range<DIM, TESS, Real, SCHEME_REF>(a.t, a.nTimeSteps, a.nStepsODE, sA, sT, start, end, h, src,
                                                     snk, c_fast, c_fb, c_sub, c_pts, nullptr, 0, &s_claim);
        __syncthreads();
        // fixed-order sum of the tile's terms: thread t takes slots t, t + blockDim, ...
        double acc = 0.0;
        for (int j = threadIdx.x; j < (int)(end - start); j += blockDim.x) acc += s_term[j];
        finish_tile(acc, tile, inst, (int)tpi, (int64_t)inst * tpi, a.partials, a.tickets, a.ll);
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

template <int TESS, typename Real>
static cudaError_t launch_register_t(const RegisterArgs &a, const LaunchCfg &cfg, cudaStream_t s)
{
    size_t smem = (size_t)(1 + TableLayout<Real>::kTParts) * a.t.nC * 6 * sizeof(Real) +
                  (size_t)a.tile_px * sizeof(double);
    auto kern = k_register_ll<TESS, Real>;
    if (smem > 48 * 1024) {
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
