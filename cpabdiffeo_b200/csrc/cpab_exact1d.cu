// cpab_exact1d.cu -- closed-form 1D integration across cell boundaries.
//
// Restates cpab/cpa1d/calcs/ClosedFormInt.py (calc_phi :64-165,
// find_crossing_time :193-256, calc_affine_phi :171-192) for a batch of
// instances on the unit interval with nC equal cells and zero-velocity
// boundary.  Inside cell c the velocity is v(x) = a x + b, so
//     x(t) = e^{a t} x + b (e^{a t} - 1) / a        (x + t b if a == 0)
// and the time to reach the cell's exit endpoint xe is
//     t = log((xe + b/a) / (x + b/a)) / a           ((xe - x)/b if a ~ 0).
// A point walks from cell to cell, consuming the remaining time, until it
// stops inside a cell or the velocity cannot carry it over the next
// endpoint (sign change / zero velocity), with the reference's 1e-16 and
// 1e-12 nudges at endpoints and its np.allclose(., 0) tests (|.| <= 1e-8).
//
// Hitting times are double in both precisions.  The FP32 mode stores the
// points in float, takes the first cell's exit time as a difference of
// logarithms (per-cell exit logarithms staged with the tables) and the
// final position's exponential in float (cf_crossing_f32, cf_phi_f32).
#include <math_constants.h>

#include "cpab_device.cuh"
#include "cpab_launch.h"

namespace cpab {

struct Exact1D {
    const double *A;  // [nC, 2] signed (a, b) of the current instance, shared memory
    const double *ba; // [nC] b / a
    const double *ia; // [nC] 1.0 / a
    const double *lx; // [2 nC] log|xn + b/a| of the cell's exit points (xn: right, then left), FP32 mode
    int nC;
    double step;      // 1/nC: vertices x_k = k*step, x_nC = 1 (np.linspace(0,1,nC+1))
};

__device__ __forceinline__ double vert(const Exact1D &e, int k) { return k == e.nC ? 1.0 : (double)k * e.step; }

__device__ __forceinline__ int cf_cell(const Exact1D &e, double x)
{
    double f = floor(x * (double)e.nC);
    f = fmin(fmax(f, 0.0), (double)(e.nC - 1));
    return (int)f;
}

__device__ __forceinline__ double cf_v(const Exact1D &e, double x, int c)
{
    if (!(0 <= x && x <= 1)) return 0.0;
    return e.A[2 * c] * x + e.A[2 * c + 1];
}

__device__ __forceinline__ bool near0(double v) { return fabs(v) <= 1e-8; }

// find_crossing_time; next = -1 for "never".
__device__ double cf_crossing(const Exact1D &e, double x, int c, int &next)
{
    const double a = e.A[2 * c], b = e.A[2 * c + 1];
    const double v = cf_v(e, x, c);
    next = -1;
    if (near0(v)) return CUDART_INF;
    const int cn = c + (v > 0 ? 1 : -1);
    if (!(0 <= cn && cn < e.nC)) return CUDART_INF;
    double xn = (v > 0) ? vert(e, cn) + 1e-16 : vert(e, c) - 1e-16;
    const double vn = cf_v(e, xn, cn);
    if (near0(vn)) return CUDART_INF;
    if ((v > 0) != (vn > 0)) return CUDART_INF;
    double t;
    if (xn == 0 || xn == 1) t = CUDART_INF;
    else if (near0(a)) t = (xn - x) / b;
    else t = e.ia[c] * log((xn + e.ba[c]) / (x + e.ba[c]));   // 1.0/a * log((xn + b/a) / (x + b/a))
    next = cn;
    return t;
}

// FP32 mode (float points; hitting times stay FP64): the time to the exit
// of the first cell as a difference of logarithms, log|xn + b/a| taken from
// the per-cell table, so that a point costs one log and no division; within
// a few ulps of the reference's log of the ratio, i.e. a time error of order
// 1e-16 |log(...)| / |a| -- far below the float result's rounding.
__device__ double cf_crossing_f32(const Exact1D &e, double x, int c, int &next)
{
    const double a = e.A[2 * c], b = e.A[2 * c + 1];
    const double v = cf_v(e, x, c);
    next = -1;
    if (near0(v)) return CUDART_INF;
    const int cn = c + (v > 0 ? 1 : -1);
    if (!(0 <= cn && cn < e.nC)) return CUDART_INF;
    const double xn = (v > 0) ? vert(e, cn) + 1e-16 : vert(e, c) - 1e-16;
    const double vn = cf_v(e, xn, cn);
    if (near0(vn)) return CUDART_INF;
    if ((v > 0) != (vn > 0)) return CUDART_INF;
    double t;
    if (xn == 0 || xn == 1) t = CUDART_INF;
    else if (near0(a)) t = (xn - x) / b;
    else t = e.ia[c] * (e.lx[2 * c + (v > 0 ? 0 : 1)] - log(fabs(x + e.ba[c])));
    next = cn;
    return t;
}

// FP32 mode: the final position x + t v(x) phi(a t), phi(z) = (e^z - 1)/z,
// with v in FP64 (it multiplies the flow's expansion e^{a t}) and phi in
// FP32 (relative error ~2e-7 of a displacement within one cell).  Equal in
// exact arithmetic to the reference's e^{at} x + b (e^{at} - 1)/a.
__device__ __forceinline__ double cf_phi_f32(const Exact1D &e, int c, double x, double t)
{
    const double a = e.A[2 * c], b = e.A[2 * c + 1];
    if (!(0 <= x && x <= 1)) return x;
    if (a == 0) return x + t * b;
    const double v = fma(a, x, b);
    const float z = (float)(a * t);
    const float phi = fabsf(z) < 1e-3f ? fmaf(z, fmaf(z, fmaf(z, 1.f / 24.f, 1.f / 6.f), 0.5f), 1.f)
                                       : expm1f(z) / z;
    return fma(t * v, (double)phi, x);
}

__device__ __forceinline__ double cf_phi(const Exact1D &e, int c, double x, double t)
{
    double a = e.A[2 * c], b = e.A[2 * c + 1];
    if (!(0 <= x && x <= 1)) { a = 0; b = 0; }
    if (a == 0) return x + t * b;
    const double ea = exp(t * a);
    return ea * x + b * (ea - 1) * e.ia[c];  // b (e^{at} - 1) / a with the cell's precomputed 1/a
}

// Every visit after the first starts at a nudged vertex (x_k + 1e-12 when
// entering cell k from the left, x_{k+1} - 1e-12 from the right), so its
// hitting time depends on (cell, direction) only.  Those are evaluated once
// per instance with the same function (cf_crossing) into shared memory, one
// record per (cell k, direction dir) at index 2 k + dir:
//   te[.] = {hitting time, entry point},
//   cn[.] = {cell of the entry point, index of the next record or -1}
// (dir 0: entered from the left, 1: from the right), so a step of the walk
// is one 16-byte and one 8-byte load.  The results are those of evaluating
// cf_crossing at every visit.
struct Transit {
    double2 *te;
    int2 *cn;
};

// Transit record entered when moving from cell c into cell n (from the left
// when moving right): 2 n + dir, or -1 when there is no next cell.
__device__ __forceinline__ int record_of(int n, int c) { return n < 0 ? -1 : 2 * n + (n > c ? 0 : 1); }

__device__ void build_transit(const Exact1D &e, Transit tr)
{
    for (int k = threadIdx.x; k < e.nC; k += blockDim.x) {
        const double x0 = fmin(1.0, fmax(0.0, vert(e, k) + 1e-12));
        const double x1 = fmin(1.0, fmax(0.0, vert(e, k + 1) - 1e-12));
        const int c0 = cf_cell(e, x0), c1 = cf_cell(e, x1);
        int n0, n1;
        const double t0 = cf_crossing(e, x0, c0, n0);
        const double t1 = cf_crossing(e, x1, c1, n1);
        tr.te[2 * k] = make_double2(t0, x0);
        tr.te[2 * k + 1] = make_double2(t1, x1);
        tr.cn[2 * k] = make_int2(c0, record_of(n0, c0));
        tr.cn[2 * k + 1] = make_int2(c1, record_of(n1, c1));
    }
}

// calc_phi for one point; returns false when the crossing cap is hit
// (the reference raises ValueError, ClosedFormInt.py:155-160).  F32: the
// first hitting time and the final position of the FP32 mode (above).
template <bool F32>
__device__ bool cf_point(const Exact1D &e, const Transit &tr, double x, double t, int cap, double &out,
                         unsigned &visits)
{
    double x_old = x, t_rem = t;
    if (0 < x_old && x_old < 1) {
        // on a vertex with non-positive velocity: start just left of it
        double u = x_old * (double)e.nC;
        int k = (int)rint(u);
        if (k >= 0 && k <= e.nC && vert(e, k) == x_old) {
            int c = k < e.nC ? k : e.nC - 1;
            double vk = e.A[2 * c] * x_old + e.A[2 * c + 1];
            if (!(vk > 0)) x_old = x_old - 1e-16;
        }
    }
    // first visit: general position
    int c = cf_cell(e, x_old), cn;
    double tc = F32 ? cf_crossing_f32(e, x_old, c, cn) : cf_crossing(e, x_old, c, cn);
    // the record of the next cell (entered at its nudged vertex, from the left when moving right)
    int idx = record_of(cn, c);
    bool ok = true;
    // walk the transit table (cheap, divergent); the final exponential runs
    // after the loop so that all lanes of a warp evaluate it together
    for (int counter = 0;;) {
        ++visits;
        // stop when the remaining time ends inside this cell, when no further
        // crossing exists (idx -1, or any index outside the table), and on NaN
        // (comparisons with NaN are false)
        if (!(tc < t_rem) || (unsigned)idx >= (unsigned)(2 * e.nC)) break;
        t_rem -= tc;
        const double2 te = tr.te[idx];
        if (++counter >= cap) {
            // the point would have been left at the crossing it just made
            x_old = te.y;
            ok = false;
            break;
        }
        const int2 nn = tr.cn[idx];
        x_old = te.y;
        tc = te.x;
        c = nn.x;
        idx = nn.y;
    }
    out = ok ? fmin(1.0, fmax(0.0, F32 ? cf_phi_f32(e, c, x_old, t_rem) : cf_phi(e, c, x_old, t_rem))) : x_old;
    return ok;
}

// Cell-sort key of a start point: only groups points (any key in [0, nC)
// keeps the results; the walk itself uses cf_cell), so float points take a
// float product and a conversion (NaN converts to 0).
__device__ __forceinline__ int sort_key(const Exact1D &e, double x) { return cf_cell(e, x); }
__device__ __forceinline__ int sort_key(const Exact1D &e, float x)
{
    return min(max((int)(x * (float)e.nC), 0), e.nC - 1);
}

// Shared memory of k_exact1d: per cell A (2 doubles), b/a and 1/a (2), the
// two exit logarithms (2), and two transit records (2 x (16 + 8) bytes) --
// 96 bytes, so what follows is 16-byte aligned -- and, when cell-sorting,
// sorted start points and results in input order [tile_pts] (Real), the
// permutation [tile_pts] (16-bit) and the histogram [nC] (int).
size_t exact1d_smem_bytes(int nC, int tile_pts, int sort, int prec)
{
    size_t b = (size_t)nC * (6 * sizeof(double) + 2 * (sizeof(double2) + sizeof(int2)));
    if (sort)
        b += 2 * (size_t)tile_pts * (prec == PREC_F64 ? sizeof(double) : sizeof(float)) +
             (size_t)tile_pts * sizeof(unsigned short) + ((size_t)nC + 2) * sizeof(int);
    return b;
}

// Resident CTAs of 256 threads the register allocation must allow per SM,
// and the tiles a CTA takes in a row.  Measured on the batched 1D workload
// (88 M points, 4096 instances), same box: 6 CTAs (40 registers) in groups
// of 2 tiles 1.98 ms; 6 CTAs, single tiles 2.02 ms; 5 CTAs (48 registers)
// 2.05 ms in groups of 2, 2.09 ms in groups of 4, 2.17 ms single; the
// compiler's own register choice (96) 2.51 ms.  A contiguous range of tiles
// per CTA (one table build per instance and CTA) was slower (3.10 ms):
// instances differ in cost, and strided groups spread them over the CTAs.
#ifndef CPAB_EXACT1D_MIN_BLOCKS
#define CPAB_EXACT1D_MIN_BLOCKS 6
#endif
#ifndef CPAB_EXACT1D_TILE_GROUP
#define CPAB_EXACT1D_TILE_GROUP 2
#endif

template <typename Real>
__global__ void __launch_bounds__(256, CPAB_EXACT1D_MIN_BLOCKS) k_exact1d(IntegrateArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nC = a.t.nC;
    double *sA = reinterpret_cast<double *>(smem_raw);
    double *s_ba = sA + 2 * nC, *s_ia = s_ba + nC, *s_lx = s_ia + nC;
    Transit tr;
    tr.te = reinterpret_cast<double2 *>(s_lx + 2 * nC);
    tr.cn = reinterpret_cast<int2 *>(tr.te + 2 * nC);
    // cell-sort scratch (see exact1d_smem_bytes)
    const int tp = a.batch.tile_pts;
    Real *s_xs = reinterpret_cast<Real *>(tr.cn + 2 * nC);
    Real *s_y = s_xs + tp;
    unsigned short *s_perm = reinterpret_cast<unsigned short *>(s_y + tp);
    // the histogram after the 16-bit permutation, rounded up to a 4-byte boundary
    int *s_hist = reinterpret_cast<int *>(s_perm + ((tp + 1) & ~1));
    __shared__ TileInfo s_tile;
    __shared__ int s_claim;
    const double T_total = a.dt * (double)a.nTimeSteps;
    const int64_t ntiles = total_tiles(a.batch);
    const int lane = threadIdx.x & 31;
    // per-lane counts stay far below 2^32 (a lane finishes a few thousand points)
    unsigned c_pts = 0, c_fail = 0, c_nan = 0;
    unsigned long long c_visits = 0;
    unsigned visits = 0;  // folded into c_visits after every tile
    int loaded = -1;
    Exact1D e;
    e.A = sA;
    e.ba = s_ba;
    e.ia = s_ia;
    e.lx = s_lx;
    e.nC = nC;
    e.step = 1.0 / (double)nC;
    // the reference gives up after nC crossings
    const int cap = nC;
    // CTAs take groups of G consecutive tiles, strided over the grid (the
    // tiles of a group mostly share an instance, so its tables are built once)
    constexpr int G = CPAB_EXACT1D_TILE_GROUP;
    for (int64_t it = 0;; ++it) {
        const int64_t grp = (int64_t)blockIdx.x + (it / G) * gridDim.x;
        const int64_t tile = grp * G + it % G;
        if (grp * G >= ntiles) break;
        if (tile >= ntiles) continue;
        if ((it & 7) == 0 && cta_cancelled(a.cancel, a.counters)) break;
        if (threadIdx.x == 0) {
            s_tile = decode_tile(a.batch, tile);
            s_claim = 0;
        }
        __syncthreads();
        const TileInfo ti = s_tile;
        if (ti.inst != loaded) {
            const double *gA = a.A + (size_t)ti.inst * nC * 2;
            for (int i = threadIdx.x; i < nC * 2; i += blockDim.x) sA[i] = gA[i];
            for (int c = threadIdx.x; c < nC; c += blockDim.x) {
                const double ac = gA[2 * c], bc = gA[2 * c + 1];
                const double ba = bc / ac;
                s_ba[c] = ba;
                s_ia[c] = 1.0 / ac;
                if (sizeof(Real) == 4) {
                    s_lx[2 * c] = log(fabs(vert(e, c + 1) + 1e-16 + ba));
                    s_lx[2 * c + 1] = log(fabs(vert(e, c) - 1e-16 + ba));
                }
            }
            __syncthreads();
            build_transit(e, tr);
            loaded = ti.inst;
            __syncthreads();
        }
        const int n = (int)(ti.end - ti.start);
        // the tile's points: 32-bit offsets from one base pointer
        const Real *tin = static_cast<const Real *>(a.pts_in) + ti.start;
        Real *tout = static_cast<Real *>(a.pts_out) + ti.start;
        if (a.sort) {
            // counting sort by start cell: a warp then takes neighbouring points,
            // which cross the same cells (same walk length).  Points are staged
            // in shared memory so that global loads and stores stay coalesced.
            for (int c = threadIdx.x; c < nC; c += blockDim.x) s_hist[c] = 0;
            __syncthreads();
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                const Real xin = tin[j];
                s_y[j] = xin;
                atomicAdd(s_hist + sort_key(e, xin), 1);
            }
            __syncthreads();
            warp0_exclusive_scan(s_hist, nC);
            __syncthreads();
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                const Real xin = s_y[j];
                const int pos = atomicAdd(s_hist + sort_key(e, xin), 1);
                s_perm[pos] = (unsigned short)j;
                s_xs[pos] = xin;
            }
            __syncthreads();
        }
        // warps claim 32 consecutive (sorted) points at a time until the tile is done
        for (;;) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&s_claim, 32);
            base = __shfl_sync(FULL, base, 0);
            if (base >= n) break;
            const int k = base + lane;
            if (k < n) {
                const Real xin = a.sort ? s_xs[k] : tin[k];
                double y;
                bool ok = cf_point<sizeof(Real) == 4>(e, tr, (double)xin, T_total, cap, y, visits);
                if (a.clamp) y = clamp_ref(y, a.clamp_lo, a.clamp_hi);
                Real yo = (Real)y;
                if (a.sort) s_y[s_perm[k]] = yo;
                else tout[k] = yo;
                ++c_pts;
                c_fail += ok ? 0u : 1u;
                c_nan += (y != y) ? 1u : 0u;
            }
        }
        c_visits += visits;
        visits = 0;
        __syncthreads();
        if (a.sort) {
            for (int j = threadIdx.x; j < n; j += blockDim.x) tout[j] = s_y[j];
            // the next tile rewrites s_y only after its first barrier
        }
    }
    if (a.counters) {
        const unsigned long long pts = warp_sum_u64(c_pts), fails = warp_sum_u64(c_fail),
                                 nans = warp_sum_u64(c_nan);
        c_visits = warp_sum_u64(c_visits);
        if ((threadIdx.x & 31) == 0) {
            if (nans) atomicAdd(a.counters + CNT_NAN, nans);
            atomicAdd(a.counters + CNT_FAST, c_visits);  // cell visits (closed-form segments)
            atomicAdd(a.counters + CNT_POINTS, pts);
            atomicAdd(a.counters + CNT_FAILED, fails);
        }
    }
}

cudaError_t launch_integrate_exact1d(const IntegrateArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s)
{
    const size_t smem = exact1d_smem_bytes(a.t.nC, a.batch.tile_pts, a.sort, prec);
    if (prec == PREC_F64) {
        auto kern = k_exact1d<double>;
        if (smem > kSmemOptInAbove) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        int grid = cfg.grid > 0 ? cfg.grid : persistent_grid(kern, cfg, smem);
        kern<<<grid, cfg.block, smem, s>>>(a);
    } else {
        auto kern = k_exact1d<float>;
        if (smem > kSmemOptInAbove) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        int grid = cfg.grid > 0 ? cfg.grid : persistent_grid(kern, cfg, smem);
        kern<<<grid, cfg.block, smem, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace cpab
