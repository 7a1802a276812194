// cpab_kernels.cu -- sm_100a kernels of the CPAB transform hot path.
//
//   k_theta_to_trels  A = B.theta for a batch of theta, then per cell
//                     signed A and Trel = expm(dt * signed A)
//                     (cpab/cpaNd/_CpaSpace.py:366-376 + _CpaCalcs.py:227-372
//                     + cpab/gpu/expm/expm_affine_by_series_{2D,3D}.py)
//   k_expm            the same from given A (no basis)
//   k_integrate       calc_T / calc_T_simple for a batch of instances
//                     (cpab/gpu/calc_2Dto2D.cu:348-445 and 1D/3D twins)
//   k_trajectory      calc_trajectory (calc_2Dto2D.cu:499-556)
//   k_cell_idx        calc_cell_idx (calc_2Dto2D.cu:323-344)
//   k_calc_v          calc_v (calc_2Dto2D.cu:561-602)
//   k_tile_prefix     tile bookkeeping for ragged batches
//
// Layout in HBM: points row-major [nPts, DIM] (the reference's layout);
// per-instance tables [N, nC, DIM*(DIM+1)] float64; the current instance's
// tables are staged in shared memory (converted to float in FP32 mode).
#include <mutex>

#include "cpab_integrate.cuh"
#include "cpab_launch.h"

namespace cpab {

// tile_prefix[i] = sum_{j<i} ceil(n_j / tile_pts); one block, sequential
// chunks per thread, then a block scan of the chunk sums.
__global__ void k_tile_prefix(const int64_t *offsets, int64_t *prefix, int N, int tile_pts)
{
    __shared__ int64_t part[1024];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int per = (N + nt - 1) / nt;
    const int b = tid * per, e = min(N, b + per);
    int64_t s = 0;
    for (int i = b; i < e; ++i) {
        int64_t n = offsets[i + 1] - offsets[i];
        s += n > 0 ? (n + tile_pts - 1) / tile_pts : 0;
    }
    part[tid] = s;
    __syncthreads();
    if (tid == 0) {
        int64_t acc = 0;
        for (int i = 0; i < nt; ++i) { int64_t v = part[i]; part[i] = acc; acc += v; }
        prefix[N] = acc;
    }
    __syncthreads();
    int64_t acc = part[tid];
    for (int i = b; i < e; ++i) {
        prefix[i] = acc;
        int64_t n = offsets[i + 1] - offsets[i];
        acc += n > 0 ? (n + tile_pts - 1) / tile_pts : 0;
    }
}

// ------------------------------------------------------------ integration

template <int DIM>
struct ArraySrc {
    const void *base;
    template <typename Real>
    __device__ __forceinline__ void load(int64_t i, PState<DIM, Real> &st) const
    {
        Real p[DIM];
        load_pt<DIM, Real>(base, i, p);
        st.set(p);
    }
};

template <int DIM>
struct ArraySnk {
    void *base;
    int clamp;
    double lo, hi;
    unsigned long long nan;
    template <typename Real>
    __device__ __forceinline__ void put(int64_t i, const PState<DIM, Real> &st)
    {
        Real p[DIM];
        st.get(p);
        bool bad = false;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            if (clamp) p[k] = clamp_ref(p[k], lo, hi);
            bad |= (p[k] != p[k]);
        }
        nan += bad ? 1 : 0;
        store_pt<DIM, Real>(base, i, p);
    }
};

template <int DIM, int TESS, typename Real, int SCHEME>
__device__ __forceinline__ void integrate_body(const IntegrateArgs &a)
{
    constexpr int NE = DIM * (DIM + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real *sA = reinterpret_cast<Real *>(smem_raw);
    Real *sT = sA + a.t.nC * NE;
    // cell-sort scratch after the tables: histogram [nC], start cells and permutation [tile_pts]
    int *s_hist = reinterpret_cast<int *>(sA + (1 + TableLayout<Real>::kTParts) * a.t.nC * NE);
    int *s_cell = s_hist + a.t.nC;
    int *s_perm = s_cell + a.batch.tile_pts;
    __shared__ TileInfo s_tile;
    __shared__ unsigned long long s_claim;

    const int tab = a.t.nC * NE;
    const Real h = (Real)(a.dt / (double)a.nStepsODE);
    const int64_t ntiles = total_tiles(a.batch);
    unsigned long long c_fast = 0, c_fb = 0, c_sub = 0, c_pts = 0;
    int loaded = -1;
    const ArraySrc<DIM> src{a.pts_in};
    ArraySnk<DIM> snk{a.pts_out, a.clamp, a.clamp_lo, a.clamp_hi, 0ull};
    ExactCross ex{nullptr, a.facets, a.nbr, a.nF, a.h_sub, a.max_crossings, 0ull, 0ull};

    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if ((((tile - blockIdx.x) / gridDim.x) & 7) == 0 && cta_cancelled(a.cancel, a.counters)) break;
        if (threadIdx.x == 0) {
            s_tile = decode_tile(a.batch, tile);
            s_claim = 0ull;
        }
        __syncthreads();
        const TileInfo ti = s_tile;
        if (ti.inst != loaded) {
            stage_tables<DIM, Real>(a.A + (size_t)ti.inst * tab, a.T + (size_t)ti.inst * tab, a.t.nC,
                                    SCHEME != SCHEME_SIMPLE, a.h_sub, sA, sT, SCHEME == SCHEME_EXACT);
            ex.A = a.A + (size_t)ti.inst * tab;
            loaded = ti.inst;
            __syncthreads();
        }
        const int64_t n = ti.end - ti.start;
        const int *perm = nullptr;
        if (a.sort) {
            // counting sort of the tile's points by start cell (order inside a cell is irrelevant:
            // every point is integrated on its own)
            for (int i = threadIdx.x; i < a.t.nC; i += blockDim.x) s_hist[i] = 0;
            __syncthreads();
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                PState<DIM, Real> st;
                src.load(ti.start + i, st);
                const int c = cell_of<DIM, TESS>(a.t, st);
                s_cell[i] = c;
                atomicAdd(s_hist + c, 1);
            }
            __syncthreads();
            warp0_exclusive_scan(s_hist, a.t.nC);
            __syncthreads();
            for (int i = threadIdx.x; i < n; i += blockDim.x) s_perm[atomicAdd(s_hist + s_cell[i], 1)] = i;
            __syncthreads();
            perm = s_perm;
        }
        // every warp works on the whole tile through the shared claim counter
        integrate_range<DIM, TESS, Real, SCHEME>(a.t, a.nTimeSteps, a.nStepsODE, sA, sT, ti.start, ti.end, h, src,
                                                 snk, c_fast, c_fb, c_sub, c_pts, perm, ti.start, &s_claim,
                                                 perm ? s_cell : nullptr, &ex);
        __syncthreads();
    }
    if (a.counters) {
        c_fast = warp_sum_u64(c_fast);
        c_fb = warp_sum_u64(c_fb);
        c_sub = warp_sum_u64(c_sub);
        c_pts = warp_sum_u64(c_pts);
        unsigned long long c_nan = warp_sum_u64(snk.nan);
        unsigned long long c_cross = 0, c_unres = 0;
        if (SCHEME == SCHEME_EXACT) {
            c_cross = warp_sum_u64(ex.crossings);
            c_unres = warp_sum_u64(ex.unresolved);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(a.counters + CNT_FAST, c_fast);
            atomicAdd(a.counters + CNT_FALLBACK, c_fb);
            atomicAdd(a.counters + CNT_SUBSTEPS, c_sub);
            atomicAdd(a.counters + CNT_POINTS, c_pts);
            if (c_nan) atomicAdd(a.counters + CNT_NAN, c_nan);
            if (c_cross) atomicAdd(a.counters + CNT_CROSSINGS, c_cross);
            if (c_unres) atomicAdd(a.counters + CNT_FAILED, c_unres);
        }
    }
}

template <int DIM, int TESS, typename Real, int SCHEME>
__global__ void __launch_bounds__(256) k_integrate(IntegrateArgs a)
{
    integrate_body<DIM, TESS, Real, SCHEME>(a);
}

// The exact scheme's exit resolution (FP64, rare) would otherwise set the
// register count of the whole kernel; the bound keeps CPAB_EXACT_MIN_BLOCKS
// CTAs of 256 threads resident per SM.
#ifndef CPAB_EXACT_MIN_BLOCKS
#define CPAB_EXACT_MIN_BLOCKS 3
#endif
template <int DIM, int TESS, typename Real>
__global__ void __launch_bounds__(256, CPAB_EXACT_MIN_BLOCKS) k_integrate_exact(IntegrateArgs a)
{
    integrate_body<DIM, TESS, Real, SCHEME_EXACT>(a);
}

// ------------------------------------------------------------ trajectory

// calc_trajectory: out is [(nTimeSteps+1), nPts, DIM]; row 0 = the input
// (the reference prepends it on the host, _CpaCalcs.py:866-868).
template <int DIM, int TESS>
__global__ void __launch_bounds__(256) k_trajectory(IntegrateArgs a, int64_t nPts)
{
    constexpr int NE = DIM * (DIM + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sA = reinterpret_cast<double *>(smem_raw);
    double *sT = sA + a.t.nC * NE;
    const int tab = a.t.nC * NE;
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        sA[i] = a.A[i];
        sT[i] = a.T[i];
    }
    __syncthreads();
    const double h = XDIV(a.dt, (double)a.nStepsODE);
    double *out = static_cast<double *>(a.pts_out);
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < nPts;
         idx += (int64_t)gridDim.x * blockDim.x) {
        double p[DIM], q[DIM];
        load_pt<DIM, double>(a.pts_in, idx, p);
        store_pt<DIM, double>(out, idx, p);
        for (int s = 0; s < a.nTimeSteps; ++s) {
            int c = exact_cell<DIM, TESS>(a.t, p);
            exact_affine<DIM>(q, sT + c * NE, p);
            if (exact_cell<DIM, TESS>(a.t, q) == c) {
#pragma unroll
                for (int i = 0; i < DIM; ++i) p[i] = q[i];
            } else {
                for (int k = 0; k < a.nStepsODE; ++k) {
                    int cc = exact_cell<DIM, TESS>(a.t, p);
                    exact_midpoint<DIM>(p, sA + cc * NE, h);
                }
            }
            store_pt<DIM, double>(out, (int64_t)(s + 1) * nPts + idx, p);
        }
    }
}

// ------------------------------------------------------------ cell index, velocity

template <int DIM, int TESS>
__global__ void k_cell_idx(Tess t, const double *pts, int32_t *out, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double p[DIM];
        load_pt<DIM, double>(pts, i, p);
        out[i] = exact_cell<DIM, TESS>(t, p);
    }
}

template <int DIM, int TESS>
__global__ void __launch_bounds__(256) k_calc_v(Tess t, const double *A, const double *pts, double *out, int64_t n)
{
    constexpr int NE = DIM * (DIM + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sA = reinterpret_cast<double *>(smem_raw);
    for (int i = threadIdx.x; i < t.nC * NE; i += blockDim.x) sA[i] = A[i];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double p[DIM], v[DIM];
        load_pt<DIM, double>(pts, i, p);
        int c = exact_cell<DIM, TESS>(t, p);
        exact_affine<DIM>(v, sA + c * NE, p);
        store_pt<DIM, double>(out, i, v);
    }
}

// ------------------------------------------------------------ expm

// expm of the 2x2 linear block, cpab/gpu/expm/expm_affine_by_series_2D.py:28-74
// (eigenvalue cases: repeated, real, complex).
__device__ void expm_2x2(double a, double b, double c, double d, double *E)
{
    double disc = (a - d) * (a - d) + 4 * b * c;
    double e = exp((a + d) / 2);
    double hd = (a - d) / 2;
    if (disc == 0) {
        E[0] = (1 + hd) * e;
        E[1] = b * e;
        E[2] = c * e;
        E[3] = (1 - hd) * e;
    } else {
        double delta, ch, s;
        if (disc > 0) {
            delta = sqrt(disc) / 2;
            ch = cosh(delta);
            s = sinh(delta) / delta;
        } else {
            delta = sqrt(-disc) / 2;
            ch = cos(delta);
            s = sin(delta) / delta;
        }
        E[0] = (ch + hd * s) * e;
        E[1] = b * s * e;
        E[2] = c * s * e;
        E[3] = (ch - hd * s) * e;
    }
}

// I + sum_{k=1..12} M^k / k! for an affine block with zero last row
// (expm_affine_by_series_2D.py:156-232, _3D.py:26-220).
template <int DIM>
__device__ void expm_taylor12(const double *M, double *T)
{
    constexpr int NC = DIM + 1, NE = DIM * NC;
    double An[NE], Bn[NE];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int c = 0; c < NC; ++c) T[r * NC + c] = (r == c) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < NE; ++k) { An[k] = M[k]; T[k] += An[k]; }
    int fact = 1;
    for (int i = 2; i <= 12; ++i) {
#pragma unroll
        for (int k = 0; k < NE; ++k) Bn[k] = An[k];
        fact *= i;
        const double inv = 1.0 / (double)fact;
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                double acc = M[r * NC] * Bn[c];
#pragma unroll
                for (int m = 1; m < DIM; ++m) acc += M[r * NC + m] * Bn[m * NC + c];
                An[r * NC + c] = acc;
            }
#pragma unroll
        for (int k = 0; k < NE; ++k) T[k] += An[k] * inv;
    }
}

// Trel for one cell from M = dt * signed A.
template <int DIM>
__device__ void affine_expm(const double *M, double *T)
{
    if (DIM == 1) {
        // cpab/cpaNd/_CpaCalcs.py:288-292
        T[0] = exp(M[0]);
        T[1] = M[1];
        if (M[0] != 0) T[1] = T[1] * (T[0] - 1) / M[0];
    } else if (DIM == 2) {
        double det = M[0] * M[4] - M[1] * M[3];
        if (det != 0) {
            double E[4];
            expm_2x2(M[0], M[1], M[3], M[4], E);
            T[0] = E[0]; T[1] = E[1]; T[3] = E[2]; T[4] = E[3];
            double i00 = M[4] / det, i11 = M[0] / det, i01 = -M[1] / det, i10 = -M[3] / det;
            double u = i00 * M[2] + i01 * M[5];
            double w = i10 * M[2] + i11 * M[5];
            T[2] = (T[0] - 1) * u + T[1] * w;
            T[5] = T[3] * u + (T[4] - 1) * w;
        } else {
            expm_taylor12<2>(M, T);
        }
    } else {
        expm_taylor12<3>(M, T);
    }
}

// signed A and Trel for n_cells = N*nC cells from A.
template <int DIM>
__global__ void k_expm(const double *A, double *signedA, double *T, int64_t n_cells, double dt, double sign)
{
    constexpr int NE = DIM * (DIM + 1);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_cells;
         c += (int64_t)gridDim.x * blockDim.x) {
        double sA[NE], M[NE], Tr[NE];
#pragma unroll
        for (int k = 0; k < NE; ++k) {
            sA[k] = sign < 0 ? -A[c * NE + k] : A[c * NE + k];
            M[k] = sA[k] * dt;
        }
        affine_expm<DIM>(M, Tr);
#pragma unroll
        for (int k = 0; k < NE; ++k) {
            if (signedA) signedA[c * NE + k] = sA[k];
            T[c * NE + k] = Tr[k];
        }
    }
}

// Per (instance, cell) after A: the sign, dt, the expm and the stores.
template <int DIM>
__device__ __forceinline__ void cell_tables(const double *a, int64_t g, double dt, double sign, double *A,
                                            double *signedA, double *T)
{
    constexpr int NE = DIM * (DIM + 1);
    double M[NE], Tr[NE];
#pragma unroll
    for (int k = 0; k < NE; ++k) {
        if (A) A[g * NE + k] = a[k];
        const double s = sign < 0 ? -a[k] : a[k];
        if (signedA) signedA[g * NE + k] = s;
        M[k] = s * dt;
    }
    affine_expm<DIM>(M, Tr);
#pragma unroll
    for (int k = 0; k < NE; ++k) T[g * NE + k] = Tr[k];
}

// A = B.theta (theta row-major [N, d], B row-major [D_A, d], rows in (cell,
// entry) order) fused with the per-cell expm.  A CTA takes 32 instances and
// a strided share of the cells: the instances' theta staged once in shared
// memory, transposed ([d][32]), then lane = instance and warp = cell, so a
// warp's B loads are one broadcast address and its theta loads one
// conflict-free row; each lane sums its dot products over j in order (the
// same operations, hence the same A, as one thread per (instance, cell)).
// Measured on 4096 theta x 100 cells (1D): the thread-per-(instance, cell)
// form took 0.12 ms, its warps' B loads spanning 32 cache lines.
constexpr int kThetaLanes = 32;
template <int DIM>
__global__ void __launch_bounds__(256) k_theta_to_trels(const double *B, const double *theta, int d, int nC, int N,
                                                        int cell_groups, double dt, double sign, double *A,
                                                        double *signedA, double *T)
{
    constexpr int NE = DIM * (DIM + 1);
    extern __shared__ double s_thT[];  // [d][kThetaLanes]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int n0 = (blockIdx.x / cell_groups) * kThetaLanes, grp = blockIdx.x % cell_groups;
    for (int e = threadIdx.x; e < kThetaLanes * d; e += blockDim.x) {
        const int i = e / d, j = e - i * d;  // consecutive e: consecutive theta of one instance
        s_thT[j * kThetaLanes + i] = (n0 + i < N) ? theta[(int64_t)(n0 + i) * d + j] : 0.0;
    }
    __syncthreads();
    const int n = n0 + lane;
    if (n >= N) return;  // no barrier follows
    for (int c = grp * nw + warp; c < nC; c += cell_groups * nw) {
        const double *Bc = B + (int64_t)c * NE * d;
        double a[NE];
#pragma unroll
        for (int k = 0; k < NE; ++k) a[k] = 0.0;
        for (int j = 0; j < d; ++j) {
            const double tj = s_thT[j * kThetaLanes + lane];
#pragma unroll
            for (int k = 0; k < NE; ++k) a[k] = fma(__ldg(Bc + k * d + j), tj, a[k]);
        }
        cell_tables<DIM>(a, (int64_t)n * nC + c, dt, sign, A, signedA, T);
    }
}

// The same with one thread per (instance, cell), for a d too large to stage
// 32 instances' theta in shared memory.
template <int DIM>
__global__ void k_theta_to_trels_cell(const double *B, const double *theta, int d, int nC, int N,
                                      double dt, double sign, double *A, double *signedA, double *T)
{
    constexpr int NE = DIM * (DIM + 1);
    const int64_t total = (int64_t)N * nC;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int n = (int)(g / nC), c = (int)(g - (int64_t)n * nC);
        const double *th = theta + (int64_t)n * d;
        const double *Bc = B + (int64_t)c * NE * d;
        double a[NE];
#pragma unroll
        for (int k = 0; k < NE; ++k) a[k] = 0.0;
        for (int j = 0; j < d; ++j) {
            const double tj = th[j];
#pragma unroll
            for (int k = 0; k < NE; ++k) a[k] = fma(Bc[k * d + j], tj, a[k]);
        }
        cell_tables<DIM>(a, g, dt, sign, A, signedA, T);
    }
}

// ------------------------------------------------------------ launchers

static int g_num_sms = 0;
int num_sms()
{
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

// Persistent grid: SMs x resident CTAs of this kernel at this block size and
// shared memory (capped by cfg.ctas_per_sm when that is smaller).
// Occupancy queries are cached per (kernel, block, shared memory) so that a
// launch inside stream capture makes no query.
int persistent_grid_impl(const void *kern, const LaunchCfg &cfg, size_t smem)
{
    struct Key {
        const void *k;
        int block;
        size_t smem;
        int per_sm;
    };
    static Key cache[64];
    static int n_cached = 0;
    static std::mutex mu;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (int i = 0; i < n_cached; ++i)
            if (cache[i].k == kern && cache[i].block == cfg.block && cache[i].smem == smem) per_sm = cache[i].per_sm;
        if (per_sm == 0) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, cfg.block, smem) != cudaSuccess ||
                per_sm < 1)
                per_sm = 1;
            if (n_cached < 64) cache[n_cached++] = Key{kern, cfg.block, smem, per_sm};
        }
    }
    if (cfg.ctas_per_sm > 0 && cfg.ctas_per_sm < per_sm) per_sm = cfg.ctas_per_sm;
    const int g = num_sms() * per_sm;
    return (cfg.max_ctas > 0 && cfg.max_ctas < g) ? cfg.max_ctas : g;
}

static int grid_for(int64_t n, int block, int per_sm = 8)
{
    int64_t g = (n + block - 1) / block;
    int64_t cap = (int64_t)num_sms() * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

template <int DIM, int TESS, typename Real, int SCHEME>
static cudaError_t launch_integrate_t(const IntegrateArgs &a, const LaunchCfg &cfg, cudaStream_t s)
{
    constexpr int NE = DIM * (DIM + 1);
    size_t smem = (size_t)(1 + TableLayout<Real>::kTParts) * a.t.nC * NE * sizeof(Real);
    if (a.sort) smem += ((size_t)a.t.nC + 2 * (size_t)a.batch.tile_pts) * sizeof(int);
    void (*kern)(IntegrateArgs);
    if constexpr (SCHEME == SCHEME_EXACT) kern = k_integrate_exact<DIM, TESS, Real>;
    else kern = k_integrate<DIM, TESS, Real, SCHEME>;
    if (smem > kSmemOptInAbove) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int grid = cfg.grid > 0 ? cfg.grid : persistent_grid(kern, cfg, smem);
    kern<<<grid, cfg.block, smem, s>>>(a);
    return cudaGetLastError();
}

template <int DIM, int TESS>
static cudaError_t launch_integrate_dt(const IntegrateArgs &a, int prec, int scheme, const LaunchCfg &cfg,
                                       cudaStream_t s)
{
    if constexpr (DIM > 1) {
        // the 2D/3D exact scheme (1D has its own kernel, k_exact1d)
        if (scheme == SCHEME_EXACT)
            return prec == PREC_F64 ? launch_integrate_t<DIM, TESS, double, SCHEME_EXACT>(a, cfg, s)
                                    : launch_integrate_t<DIM, TESS, float, SCHEME_EXACT>(a, cfg, s);
    }
    if (prec == PREC_F64) {
        if (scheme == SCHEME_REF) return launch_integrate_t<DIM, TESS, double, SCHEME_REF>(a, cfg, s);
        return launch_integrate_t<DIM, TESS, double, SCHEME_SIMPLE>(a, cfg, s);
    }
    if (scheme == SCHEME_REF) return launch_integrate_t<DIM, TESS, float, SCHEME_REF>(a, cfg, s);
    return launch_integrate_t<DIM, TESS, float, SCHEME_SIMPLE>(a, cfg, s);
}

cudaError_t launch_integrate(const IntegrateArgs &a, int prec, int scheme, const LaunchCfg &cfg, cudaStream_t s)
{
    const int dim = a.t.dim, tess = a.t.tess;
    if (dim == 1) return launch_integrate_dt<1, 2>(a, prec, scheme, cfg, s);
    if (dim == 2) return tess == 1 ? launch_integrate_dt<2, 1>(a, prec, scheme, cfg, s)
                                   : launch_integrate_dt<2, 2>(a, prec, scheme, cfg, s);
    return tess == 1 ? launch_integrate_dt<3, 1>(a, prec, scheme, cfg, s)
                     : launch_integrate_dt<3, 2>(a, prec, scheme, cfg, s);
}

cudaError_t launch_tile_prefix(const int64_t *offsets, int64_t *prefix, int N, int tile_pts, cudaStream_t s)
{
    k_tile_prefix<<<1, 1024, 0, s>>>(offsets, prefix, N, tile_pts);
    return cudaGetLastError();
}

template <int DIM, int TESS>
static cudaError_t launch_traj_t(const IntegrateArgs &a, int64_t nPts, cudaStream_t s)
{
    constexpr int NE = DIM * (DIM + 1);
    size_t smem = (size_t)2 * a.t.nC * NE * sizeof(double);
    auto kern = k_trajectory<DIM, TESS>;
    if (smem > kSmemOptInAbove) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<grid_for(nPts, 256, 4), 256, smem, s>>>(a, nPts);
    return cudaGetLastError();
}

cudaError_t launch_trajectory(const IntegrateArgs &a, int64_t nPts, cudaStream_t s)
{
    const int dim = a.t.dim, tess = a.t.tess;
    if (dim == 1) return launch_traj_t<1, 2>(a, nPts, s);
    if (dim == 2) return tess == 1 ? launch_traj_t<2, 1>(a, nPts, s) : launch_traj_t<2, 2>(a, nPts, s);
    return tess == 1 ? launch_traj_t<3, 1>(a, nPts, s) : launch_traj_t<3, 2>(a, nPts, s);
}

cudaError_t launch_cell_idx(const Tess &t, const double *pts, int32_t *out, int64_t n, cudaStream_t s)
{
    int g = grid_for(n, 256);
    if (t.dim == 1) k_cell_idx<1, 2><<<g, 256, 0, s>>>(t, pts, out, n);
    else if (t.dim == 2) {
        if (t.tess == 1) k_cell_idx<2, 1><<<g, 256, 0, s>>>(t, pts, out, n);
        else k_cell_idx<2, 2><<<g, 256, 0, s>>>(t, pts, out, n);
    } else {
        if (t.tess == 1) k_cell_idx<3, 1><<<g, 256, 0, s>>>(t, pts, out, n);
        else k_cell_idx<3, 2><<<g, 256, 0, s>>>(t, pts, out, n);
    }
    return cudaGetLastError();
}

template <int DIM, int TESS>
static cudaError_t launch_v_t(const Tess &t, const double *A, const double *pts, double *out, int64_t n,
                              cudaStream_t s)
{
    constexpr int NE = DIM * (DIM + 1);
    size_t smem = (size_t)t.nC * NE * sizeof(double);
    auto kern = k_calc_v<DIM, TESS>;
    if (smem > kSmemOptInAbove) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<grid_for(n, 256, 4), 256, smem, s>>>(t, A, pts, out, n);
    return cudaGetLastError();
}

cudaError_t launch_calc_v(const Tess &t, const double *A, const double *pts, double *out, int64_t n, cudaStream_t s)
{
    if (t.dim == 1) return launch_v_t<1, 2>(t, A, pts, out, n, s);
    if (t.dim == 2) return t.tess == 1 ? launch_v_t<2, 1>(t, A, pts, out, n, s) : launch_v_t<2, 2>(t, A, pts, out, n, s);
    return t.tess == 1 ? launch_v_t<3, 1>(t, A, pts, out, n, s) : launch_v_t<3, 2>(t, A, pts, out, n, s);
}

cudaError_t launch_expm(int dim, const double *A, double *signedA, double *T, int64_t n_cells, double dt, double sign,
                        cudaStream_t s)
{
    int g = grid_for(n_cells, 128);
    if (dim == 1) k_expm<1><<<g, 128, 0, s>>>(A, signedA, T, n_cells, dt, sign);
    else if (dim == 2) k_expm<2><<<g, 128, 0, s>>>(A, signedA, T, n_cells, dt, sign);
    else k_expm<3><<<g, 128, 0, s>>>(A, signedA, T, n_cells, dt, sign);
    return cudaGetLastError();
}

template <int DIM>
static cudaError_t launch_theta_to_trels_t(const double *B, const double *theta, int d, int nC, int N, double dt,
                                           double sign, double *A, double *signedA, double *T, cudaStream_t s)
{
    if (N <= 0 || nC <= 0) return cudaGetLastError();
    const size_t smem = (size_t)kThetaLanes * d * sizeof(double);
    if (smem <= 100 * 1024) {
        if (smem > kSmemOptInAbove) {
            cudaError_t e = cudaFuncSetAttribute(k_theta_to_trels<DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
        }
        // about four CTAs per SM: the instance blocks times a split of the cells
        const int blocks = (N + kThetaLanes - 1) / kThetaLanes;
        const int max_groups = (nC + 7) / 8;  // 8 warps per CTA
        const int want = (4 * num_sms() + blocks - 1) / blocks;
        const int groups = std::max(1, std::min(want, max_groups));
        k_theta_to_trels<DIM><<<blocks * groups, 256, smem, s>>>(B, theta, d, nC, N, groups, dt, sign, A, signedA, T);
    } else {
        const int g = grid_for((int64_t)N * nC, 128);
        k_theta_to_trels_cell<DIM><<<g, 128, 0, s>>>(B, theta, d, nC, N, dt, sign, A, signedA, T);
    }
    return cudaGetLastError();
}

cudaError_t launch_theta_to_trels(int dim, const double *B, const double *theta, int d, int nC, int N, double dt,
                                  double sign, double *A, double *signedA, double *T, cudaStream_t s)
{
    if (dim == 1) return launch_theta_to_trels_t<1>(B, theta, d, nC, N, dt, sign, A, signedA, T, s);
    if (dim == 2) return launch_theta_to_trels_t<2>(B, theta, d, nC, N, dt, sign, A, signedA, T, s);
    return launch_theta_to_trels_t<3>(B, theta, d, nC, N, dt, sign, A, signedA, T, s);
}

}  // namespace cpab
