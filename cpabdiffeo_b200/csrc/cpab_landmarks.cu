// cpab_landmarks.cu -- batched Gaussian landmark log-likelihood.
//
// For N instances (signed tables of calc_T_fwd) and landmark pairs
// (src_i, dst_i), i < n_lm:
//     ll[n] = sum_i -0.5 |T_n(src_i) - dst_i|^2 / sigma^2
// which is calc_T_fwd of the landmarks followed by calc_err_per_sample and
// calc_ll_per_sample (cpab/cpa2d/model/transformations/landmarks/
// _ScaleDependentLogLikelihoodGaussian.py:29-73, gpu/gaussian.py:12-22; the
// 1D twin cpab/cpa1d/model/transformations/landmarks/gpu/gaussian.py:17-20),
// summed (_ScaleDependentLogLikelihoodGeneral.__call__).  The integration is
// the reference scheme through the shared lane scheduler; the per-landmark
// terms go to shared memory and are summed in a fixed order per tile, tiles
// per instance in index order, so results do not depend on the batch.
#include "cpab_integrate.cuh"
#include "cpab_landmarks.h"
#include "cpab_launch.h"
#include "cpab_reduce.cuh"

namespace cpab {

namespace {

// Start points: the instance's landmarks (double [n_lm, DIM]).
template <int DIM>
struct LandmarkSrc {
    const double *src;  // this instance's first landmark
    int64_t base;       // global index of that landmark
    template <typename Real>
    __device__ __forceinline__ void load(int64_t i, PState<DIM, Real> &st) const
    {
        double p[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) p[k] = __ldg(src + (i - base) * DIM + k);
        st.set(p);
    }
};

// End points: the Gaussian term into the tile's shared-memory slot, and the
// transformed landmark when asked for.
template <int DIM>
struct LandmarkSnk {
    const double *dst;
    double *transformed;  // this instance's first transformed landmark, or nullptr
    int64_t base, tile_start;
    double k;             // -0.5 / sigma^2
    double *term;
    int clamp;
    double lo, hi;
    template <typename Real>
    __device__ __forceinline__ void put(int64_t i, const PState<DIM, Real> &st)
    {
        const int64_t j = i - base;
        double x[DIM];
        st.get(x);
        if (clamp) {
            // calc_T's end-point clamp (threshold_krnl)
#pragma unroll
            for (int d = 0; d < DIM; ++d) x[d] = clamp_ref(x[d], lo, hi);
        }
        double e2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const double e = x[d] - __ldg(dst + j * DIM + d);
            e2 += e * e;
            if (transformed) transformed[j * DIM + d] = x[d];
        }
        term[i - tile_start] = k * e2;
    }
};

template <int DIM, int TESS, typename Real>
__global__ void __launch_bounds__(256) k_landmark_ll(LandmarkArgs a)
{
    constexpr int NE = DIM * (DIM + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real *sA = reinterpret_cast<Real *>(smem_raw);
    Real *sT = sA + a.t.nC * NE;
    // per-landmark terms of the current tile, after the tables (a multiple of 8 bytes)
    double *s_term = reinterpret_cast<double *>(sA + (1 + TableLayout<Real>::kTParts) * a.t.nC * NE);
    __shared__ unsigned long long s_claim;
    const int tab = a.t.nC * NE;
    const Real h = (Real)(a.dt / (double)a.nStepsODE);
    const int64_t tpi = ((int64_t)a.n_lm + a.tile_pts - 1) / a.tile_pts;
    const int64_t ntiles = tpi * a.N;
    const double k = -0.5 / (a.sigma * a.sigma);
    unsigned long long c_fast = 0, c_fb = 0, c_sub = 0, c_pts = 0;
    int loaded = -1;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if ((((tile - blockIdx.x) / gridDim.x) & 7) == 0 && cta_cancelled(a.cancel, a.counters)) break;
        const int inst = (int)(tile / tpi);
        const int64_t kt = tile - (int64_t)inst * tpi;
        const int64_t base = (int64_t)inst * a.n_lm;
        const int64_t start = base + kt * a.tile_pts;
        const int64_t end = min(start + (int64_t)a.tile_pts, base + a.n_lm);
        if (inst != loaded) {
            __syncthreads();
            stage_tables<DIM, Real>(a.A + (size_t)inst * tab, a.T + (size_t)inst * tab, a.t.nC, true,
                                    a.h_sub, sA, sT);
            loaded = inst;
        }
        LandmarkSrc<DIM> src{a.src + (int64_t)inst * a.src_stride * DIM, base};
        LandmarkSnk<DIM> snk{a.dst + (int64_t)inst * a.dst_stride * DIM,
                             a.transformed ? a.transformed + base * DIM : nullptr,
                             base, start, k, s_term, a.clamp, a.clamp_lo, a.clamp_hi};
        if (threadIdx.x == 0) s_claim = 0ull;
        __syncthreads();
        integrate_range<DIM, TESS, Real, SCHEME_REF>(a.t, a.nTimeSteps, a.nStepsODE, sA, sT, start, end, h, src,
                                                     snk, c_fast, c_fb, c_sub, c_pts, nullptr, 0, &s_claim);
        __syncthreads();
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

template <int DIM, int TESS, typename Real>
cudaError_t launch_t(const LandmarkArgs &a, const LaunchCfg &cfg, cudaStream_t s)
{
    const size_t smem = landmark_smem_bytes(a.t, a.tile_pts, sizeof(Real) == 8 ? PREC_F64 : PREC_F32);
    auto kern = k_landmark_ll<DIM, TESS, Real>;
    if (smem > kSmemOptInAbove) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int64_t ntiles = (((int64_t)a.n_lm + a.tile_pts - 1) / a.tile_pts) * a.N;
    int64_t grid = persistent_grid(kern, cfg, smem);
    if (grid > ntiles) grid = ntiles;
    kern<<<(unsigned)grid, cfg.block, smem, s>>>(a);
    return cudaGetLastError();
}

template <int DIM, int TESS>
cudaError_t launch_dt(const LandmarkArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s)
{
    return prec == PREC_F64 ? launch_t<DIM, TESS, double>(a, cfg, s) : launch_t<DIM, TESS, float>(a, cfg, s);
}

}  // namespace

size_t landmark_smem_bytes(const Tess &t, int tile_pts, int prec)
{
    const int ne = t.dim * (t.dim + 1);
    const size_t tables = prec == PREC_F64 ? (size_t)t.nC * ne * 2 * 8 : (size_t)t.nC * ne * 2 * 4;
    return tables + (size_t)tile_pts * sizeof(double);
}

cudaError_t launch_landmark_ll(const LandmarkArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s)
{
    switch (a.t.dim * 10 + a.t.tess) {
    case 11:
    case 12: return launch_dt<1, 2>(a, prec, cfg, s);
    case 21: return launch_dt<2, 1>(a, prec, cfg, s);
    case 22: return launch_dt<2, 2>(a, prec, cfg, s);
    case 31: return launch_dt<3, 1>(a, prec, cfg, s);
    case 32: return launch_dt<3, 2>(a, prec, cfg, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace cpab
