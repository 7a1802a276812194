// cpab_register3d.cu -- trilinear remap of volumes and the 3D Gaussian
// registration likelihood.
//
//   k_remap3d_ssd     warped = trilinear(src, map) for N volumes [H, W, D]
//                     indexed [row][col][slice] -- the order of the reference's
//                     dense 3D grid, np.mgrid[0:Ny, 0:Nx, 0:Nz] with z fastest
//                     (cpab/cpa3d/calcs/_CpaCalcs.py:45-76) -- sampled at map
//                     points (x, y, z) = (column, row, slice), zero outside
//                     (remap3d of cpab/cpa3d/TransformWrapper.py:230-286), and
//                     optionally ll = sum -0.5 (warped - dst)^2 / sigma^2.
//   k_register3d_ll   the same likelihood fused with calc_T of every voxel
//                     centre ((c+0.5)/W, (r+0.5)/H, (k+0.5)/D) of the unit
//                     cube (the 3D form of the 2D registration likelihood,
//                     cpab/cpa2d/model/transformations/register/
//                     _ScaleDependentLogLikelihoodGaussian.py:34-109); the
//                     transformed points are never stored.
// Sums are deterministic (cpab_reduce.cuh).
#include "cpab_integrate.cuh"
#include "cpab_launch.h"
#include "cpab_reduce.cuh"
#include "cpab_register3d.h"

namespace cpab {

namespace {

// Trilinear sample at voxel coordinates (px, py, pz): floor and fractions in
// double (floor by adding 1.5 * 2^52 rounding toward -inf, no conversion
// instruction), taps combined along x, then y, then z, in the map's / the
// likelihood's precision.
struct Taps3 {
    float v[8];      // (dz, dy, dx) in bit order k = 4 dz + 2 dy + dx
    double fx, fy, fz;
    bool in;
};

__device__ __forceinline__ void taps3_issue(const float *img, int H, int W, int D, double px, double py, double pz,
                                            Taps3 &t)
{
    constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
    const double sx = __dadd_rd(px, kRound), sy = __dadd_rd(py, kRound), sz = __dadd_rd(pz, kRound);
    const double fx0 = sx - kRound, fy0 = sy - kRound, fz0 = sz - kRound;
    t.in = fx0 > -2.0 && fx0 < (double)W + 1.0 && fy0 > -2.0 && fy0 < (double)H + 1.0 && fz0 > -2.0 &&
           fz0 < (double)D + 1.0;  // false for NaN
    t.fx = px - fx0;
    t.fy = py - fy0;
    t.fz = pz - fz0;
    const int c0 = t.in ? __double2loint(sx) : -2, r0 = t.in ? __double2loint(sy) : -2;
    const int k0 = t.in ? __double2loint(sz) : -2;
    if (c0 >= 0 && c0 + 1 < W && r0 >= 0 && r0 + 1 < H && k0 >= 0 && k0 + 1 < D) {
        const float *q = img + ((int64_t)r0 * W + c0) * D + k0;
        const int64_t sr = (int64_t)W * D;
#pragma unroll
        for (int k = 0; k < 8; ++k) t.v[k] = __ldg(q + ((k >> 1) & 1) * sr + (k & 1) * D + (k >> 2));
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int c = c0 + (k & 1), r = r0 + ((k >> 1) & 1), z = k0 + (k >> 2);
            t.v[k] = (r >= 0 && r < H && c >= 0 && c < W && z >= 0 && z < D)
                         ? __ldg(img + ((int64_t)r * W + c) * D + z)
                         : 0.0f;
        }
    }
}

template <typename Real>
__device__ __forceinline__ Real taps3_combine(const Taps3 &t);

template <>
__device__ __forceinline__ double taps3_combine<double>(const Taps3 &t)
{
    if (!t.in) return 0.0;
    double v[2];
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
        const float *q = t.v + 4 * dz;
        const double top = (1 - t.fx) * (double)q[0] + t.fx * (double)q[1];
        const double bot = (1 - t.fx) * (double)q[2] + t.fx * (double)q[3];
        v[dz] = (1 - t.fy) * top + t.fy * bot;
    }
    return (1 - t.fz) * v[0] + t.fz * v[1];
}

template <>
__device__ __forceinline__ float taps3_combine<float>(const Taps3 &t)
{
    if (!t.in) return 0.0f;
    const float wx = (float)t.fx, wy = (float)t.fy, wz = (float)t.fz;
    float v[2];
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
        const float *q = t.v + 4 * dz;
        const float top = fmaf(wx, q[1] - q[0], q[0]);
        const float bot = fmaf(wx, q[3] - q[2], q[2]);
        v[dz] = fmaf(wy, bot - top, top);
    }
    return fmaf(wz, v[1] - v[0], v[0]);
}

template <typename Real>
__device__ __forceinline__ Real trilinear(const float *img, int H, int W, int D, double px, double py, double pz)
{
    Taps3 t;
    taps3_issue(img, H, W, D, px, py, pz, t);
    return taps3_combine<Real>(t);
}

// One voxel per thread and iteration, voxels in increasing order per thread.
template <typename MapT>
__global__ void __launch_bounds__(256) k_remap3d_ssd(Remap3dArgs a)
{
    const int inst = blockIdx.y;
    const int64_t nvx = (int64_t)a.H * a.W * a.D;
    const int64_t tile = blockIdx.x;
    const int64_t start = tile * a.tile_px;
    const int n = (int)(min(start + (int64_t)a.tile_px, nvx) - start);
    const int64_t off = (int64_t)inst * nvx + start;
    const MapT *map = static_cast<const MapT *>(a.map) + 3 * off;
    const float *src = a.src + (int64_t)inst * nvx;
    const float *dst = a.dst ? a.dst + off : nullptr;
    float *warped = a.warped ? a.warped + off : nullptr;
    const double k = -0.5 / (a.sigma * a.sigma);
    double acc = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const MapT w = trilinear<MapT>(src, a.H, a.W, a.D, (double)map[3 * j] * a.sx + a.ox,
                                       (double)map[3 * j + 1] * a.sy + a.oy, (double)map[3 * j + 2] * a.sz + a.oz);
        if (warped) warped[j] = (float)w;
        if (dst) {
            const double e = (double)w - (double)__ldg(dst + j);
            acc += e * e * k;
        }
    }
    if (dst) {
        const int tpi = (int)gridDim.x;
        finish_tile(acc, (int64_t)inst * tpi + tile, inst, tpi, (int64_t)inst * tpi, a.partials, a.tickets, a.ll);
    }
}

// Start and end points of the current tile's voxels live in shared memory,
// three doubles per voxel: a convergent pass writes the voxel centres
// ((col+0.5)/W, (row+0.5)/H, (dep+0.5)/D) of voxels j = (row * W + col) * D
// + dep, the lane loop takes a point's start from its slot and writes its
// end point back, and a second convergent pass samples src there, compares
// with dst and sums the terms in a fixed order (thread t: voxels t,
// t + blockDim, ...).  Index arithmetic and sampling stay out of the lane
// loop, whose register count sets the CTAs per SM.
struct SlotSrc3 {
    const double *slot;
    int64_t tile_start;
    template <typename Real>
    __device__ __forceinline__ void load(int64_t i, PState<3, Real> &st) const
    {
        const double *v = slot + 3 * (i - tile_start);
        const double p[3] = {v[0], v[1], v[2]};
        st.set(p);
    }
};

struct SlotSnk3 {
    double *slot;
    int64_t tile_start;
    template <typename Real>
    __device__ __forceinline__ void put(int64_t i, const PState<3, Real> &st)
    {
        double p[3];
        st.get(p);
        double *v = slot + 3 * (i - tile_start);
        v[0] = p[0];
        v[1] = p[1];
        v[2] = p[2];
    }
};

template <int TESS, typename Real>
__global__ void __launch_bounds__(256) k_register3d_ll(Register3dArgs a)
{
    constexpr int DIM = 3, NE = 12;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real *sA = reinterpret_cast<Real *>(smem_raw);
    Real *sT = sA + a.t.nC * NE;
    double *s_pos = reinterpret_cast<double *>(sA + (1 + TableLayout<Real>::kTParts) * a.t.nC * NE);
    double *s_grp = s_pos + 3 * (size_t)a.tile_px;  // 32-voxel group sums of the likelihood
    __shared__ unsigned long long s_claim;
    const int tab = a.t.nC * NE;
    const Real h = (Real)(a.dt / (double)a.nStepsODE);
    const int64_t nvx = (int64_t)a.H * a.W * a.D;
    const int64_t tpi = (nvx + a.tile_px - 1) / a.tile_px;
    const int64_t ntiles = tpi * a.N;
    const int cpi = (int)((nvx + kSumChunk - 1) / kSumChunk);  // chunk partials per volume
    unsigned long long c_fast = 0, c_fb = 0, c_sub = 0, c_pts = 0;
    int loaded = -1;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if ((((tile - blockIdx.x) / gridDim.x) & 7) == 0 && cta_cancelled(a.cancel, a.counters)) break;
        const int inst = (int)(tile / tpi);
        const int64_t kt = tile - (int64_t)inst * tpi;
        const int64_t base = (int64_t)inst * nvx;
        const int64_t j0 = kt * a.tile_px;  // first voxel of the tile in its volume
        const int64_t start = base + j0;
        const int n = (int)(min(start + (int64_t)a.tile_px, base + nvx) - start);
        if (inst != loaded) {
            __syncthreads();
            stage_tables<DIM, Real>(a.A + (size_t)inst * tab, a.T + (size_t)inst * tab, a.t.nC, true,
                                    a.h_sub, sA, sT);
            loaded = inst;
        }
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int64_t q = j0 + j, rc = q / a.D, dep = q - rc * a.D;
            const int64_t r = rc / a.W, c = rc - r * a.W;
            double *v = s_pos + 3 * j;
            v[0] = ((double)c + 0.5) / (double)a.W;
            v[1] = ((double)r + 0.5) / (double)a.H;
            v[2] = ((double)dep + 0.5) / (double)a.D;
        }
        if (threadIdx.x == 0) s_claim = 0ull;
        __syncthreads();
        const SlotSrc3 src{s_pos, start};
        SlotSnk3 snk{s_pos, start};
        integrate_range<DIM, TESS, Real, SCHEME_REF>(a.t, a.nTimeSteps, a.nStepsODE, sA, sT, start, start + n, h,
                                                     src, snk, c_fast, c_fb, c_sub, c_pts, nullptr, 0, &s_claim);
        __syncthreads();
        const float *img = a.src + base, *ref = a.dst + base;
        float *warped = a.warped ? a.warped + base : nullptr;
        const double k = -0.5 / (a.sigma * a.sigma);
        // each voxel's term replaces the first coordinate of its slot, then the chunk-ordered sum
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            double *v = s_pos + 3 * j;
            const Real w = trilinear<Real>(img, a.H, a.W, a.D, v[0] * a.W - 0.5, v[1] * a.H - 0.5, v[2] * a.D - 0.5);
            if (warped) warped[j0 + j] = (float)w;
            const double e = (double)w - (double)__ldg(ref + j0 + j);
            v[0] = __dmul_rn(__dmul_rn(e, e), k);
        }
        __syncthreads();
        finish_tile_chunks(n, [&](int j) { return s_pos[3 * j]; }, s_grp, (int64_t)inst * cpi + j0 / kSumChunk, inst,
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

template <int TESS, typename Real>
cudaError_t launch_register3d_t(const Register3dArgs &a, const LaunchCfg &cfg, cudaStream_t s)
{
    const size_t smem = register3d_smem_bytes(a.t.nC, a.tile_px, sizeof(Real) == 8 ? PREC_F64 : PREC_F32);
    auto kern = k_register3d_ll<TESS, Real>;
    if (smem > kSmemOptInAbove) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int64_t nvx = (int64_t)a.H * a.W * a.D;
    const int64_t ntiles = ((nvx + a.tile_px - 1) / a.tile_px) * a.N;
    int64_t grid = persistent_grid(kern, cfg, smem);
    if (grid > ntiles) grid = ntiles;
    kern<<<(unsigned)grid, cfg.block, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

size_t register3d_smem_bytes(int nC, int tile_px, int prec)
{
    const size_t tables = prec == PREC_F64 ? (size_t)nC * 12 * 2 * 8 : (size_t)nC * 12 * 2 * 4;
    // three doubles per voxel slot, then the 32-voxel group sums
    return tables + (size_t)tile_px * 3 * sizeof(double) + (size_t)((tile_px + 31) / 32) * sizeof(double);
}

cudaError_t launch_remap3d_ssd(const Remap3dArgs &a, int map_prec, cudaStream_t s)
{
    const int64_t nvx = (int64_t)a.H * a.W * a.D;
    dim3 grid((unsigned)((nvx + a.tile_px - 1) / a.tile_px), (unsigned)a.N);
    if (map_prec == PREC_F64) k_remap3d_ssd<double><<<grid, 256, 0, s>>>(a);
    else k_remap3d_ssd<float><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_register3d_ll(const Register3dArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s)
{
    if (a.t.tess == 1)
        return prec == PREC_F64 ? launch_register3d_t<1, double>(a, cfg, s) : launch_register3d_t<1, float>(a, cfg, s);
    return prec == PREC_F64 ? launch_register3d_t<2, double>(a, cfg, s) : launch_register3d_t<2, float>(a, cfg, s);
}

}  // namespace cpab
