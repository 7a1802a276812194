// cpab_device.cuh -- device helpers shared by the kernel files: point
// I/O, tile decoding of (ragged) batches, warp reductions, the 1D clamp.
#pragma once

#include "cpab_internal.h"

namespace cpab {

constexpr unsigned FULL = 0xffffffffu;

// ------------------------------------------------------------ points I/O

template <int DIM, typename Real>
__device__ __forceinline__ void load_pt(const void *base, int64_t i, Real *p)
{
    const Real *b = static_cast<const Real *>(base) + i * DIM;
#pragma unroll
    for (int k = 0; k < DIM; ++k) p[k] = __ldg(b + k);
}

template <int DIM, typename Real>
__device__ __forceinline__ void store_pt(void *base, int64_t i, const Real *p)
{
    Real *b = static_cast<Real *>(base) + i * DIM;
#pragma unroll
    for (int k = 0; k < DIM; ++k) b[k] = p[k];
}

// threshold_krnl of cpab/cpaNd/_CpaSpace.py:35-43.
template <typename Real>
__device__ __forceinline__ Real clamp_ref(Real a, double lo, double hi)
{
    if (a < (Real)lo) return (Real)lo;
    if (a > (Real)hi) return (Real)hi;
    return a;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    return v;
}

// ------------------------------------------------------------ tiles

struct TileInfo {
    int inst;
    int64_t start, end;
};

__device__ __forceinline__ int64_t total_tiles(const Batch &b)
{
    return b.tile_prefix ? b.tile_prefix[b.N] : (int64_t)b.N * b.tiles_per_inst;
}

__device__ __forceinline__ TileInfo decode_tile(const Batch &b, int64_t tile)
{
    TileInfo ti;
    if (!b.tile_prefix) {
        int64_t inst = tile / b.tiles_per_inst;
        int64_t k = tile - inst * b.tiles_per_inst;
        ti.inst = (int)inst;
        int64_t base = inst * b.n_uniform;
        ti.start = base + k * b.tile_pts;
        int64_t e = ti.start + b.tile_pts, lim = base + b.n_uniform;
        ti.end = e < lim ? e : lim;
        return ti;
    }
    // first index with prefix > tile, minus one (skips empty instances)
    int lo = 0, hi = b.N;  // prefix[0] = 0 <= tile < prefix[N]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (b.tile_prefix[mid] <= tile) lo = mid; else hi = mid;
    }
    ti.inst = lo;
    ti.start = b.offsets[lo] + (tile - b.tile_prefix[lo]) * b.tile_pts;
    int64_t e = ti.start + b.tile_pts, lim = b.offsets[lo + 1];
    ti.end = e < lim ? e : lim;
    return ti;
}

// True (in every thread of the CTA) once the context's cancel flag is set;
// call at a point all threads reach.  The persistent kernels poll it every
// 8th tile (the flag is in device memory: an L2 read).
__device__ __forceinline__ bool cta_cancelled(const volatile int *flag, unsigned long long *counters)
{
    __shared__ int s_stop;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_stop = (flag && *flag) ? 1 : 0;
        if (s_stop && counters) atomicAdd(counters + CNT_CANCELLED, 1ull);
    }
    __syncthreads();
    return s_stop != 0;
}

// Exclusive prefix sum of hist[0, n) in place, by the CTA's first warp
// (each lane scans a contiguous chunk, the chunk totals are combined with
// shuffles).  The caller synchronises before and after.
__device__ __forceinline__ void warp0_exclusive_scan(int *hist, int n)
{
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const int per = (n + 31) / 32;
    const int lo = min(lane * per, n), hi = min(lo + per, n);
    int sum = 0;
    for (int c = lo; c < hi; ++c) sum += hist[c];
    int inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, inc, o);
        if (lane >= o) inc += v;
    }
    int run = inc - sum;
    for (int c = lo; c < hi; ++c) {
        const int v = hist[c];
        hist[c] = run;
        run += v;
    }
}

}  // namespace cpab
