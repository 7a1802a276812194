// cpab_reduce.cuh -- deterministic per-instance sums over tiles: each CTA
// reduces its tile in a fixed lane / warp order, stores the tile's partial,
// and the last tile of an instance to finish (atomic ticket with fences) adds
// that instance's partials in index order.  A result is therefore the same
// alone and inside any batch, whatever the launch shape.
#pragma once

#include "cpab_device.cuh"

namespace cpab {

__device__ __forceinline__ double warp_sum_f64(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    return v;
}

// Reduce `acc` over the CTA (fixed order) and hand the tile's partial to the
// per-image bookkeeping.  All threads of the CTA must call this.
__device__ __forceinline__ void finish_tile(double acc, int64_t tile, int inst, int tiles_of_inst, int64_t first_tile_of_inst,
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

// finish_tile for CTAs that loop over tiles: the same sums, with one barrier
// instead of two.  Thread 0 stores the tile's partial and takes the ticket
// after the barrier while the other warps go on with the next tile; the warp
// sums are double-buffered by tile parity, so a buffer is written again only
// after the next barrier, which thread 0 reaches once it is done reading.
__device__ __forceinline__ void finish_tile_overlapped(double acc, int parity, int64_t tile, int inst,
                                                       int tiles_of_inst, int64_t first_tile_of_inst,
                                                       double *partials, unsigned *tickets, double *ll_out)
{
    __shared__ double s_w2[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    acc = warp_sum_f64(acc);
    if (lane == 0) s_w2[parity][warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += s_w2[parity][w];
        partials[tile] = s;
        __threadfence();
        const unsigned ticket = atomicAdd(tickets + inst, 1u);
        if (ticket == (unsigned)tiles_of_inst - 1u) {
            __threadfence();
            double tot = 0.0;
            for (int k = 0; k < tiles_of_inst; ++k) tot += ((volatile double *)partials)[first_tile_of_inst + k];
            ll_out[inst] = tot;
            tickets[inst] = 0u;  // ready for the next call
        }
    }
}

// The tile's partial only (fixed lane / warp order, one barrier, warp sums
// double-buffered by tile parity as above): for kernels whose per-instance
// sums are finished by sum_partials_in_order afterwards, so no fence or
// atomic sits in the tile loop.
__device__ __forceinline__ void store_tile_partial(double acc, int parity, int64_t tile, double *partials)
{
    __shared__ double s_w3[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    acc = warp_sum_f64(acc);
    if (lane == 0) s_w3[parity][warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += s_w3[parity][w];
        partials[tile] = s;
    }
}

// Points per chunk partial of finish_tile_chunks (eight groups of 32).
constexpr int kSumChunk = 256;

// Chunk-ordered sums for the fused likelihood kernels, whose tiles start at
// multiples of kSumChunk within their instance.  term(j) is the j-th point
// of the tile (j < n).  Each warp reduces groups of 32 consecutive points
// with a fixed shuffle tree (s_grp: n/32 rounded up doubles of shared
// memory); each chunk of 256 points adds its group sums in point order and
// stores the chunk partial at partials[first_chunk + c]; the last tile of the
// instance to finish (atomic ticket with fences) adds the instance's chunk
// partials in a fixed order (32 strided sums, then a shuffle tree).  The result depends on the points' terms only --
// not on the tile size, the block size or the batch -- so a launch may pick
// its tile size freely.  All threads of the CTA must call this.
template <class Term>
__device__ __forceinline__ void finish_tile_chunks(int n, const Term &term, double *s_grp, int64_t first_chunk,
                                                   int inst, int tiles_of_inst, int chunks_of_inst,
                                                   double *partials, unsigned *tickets, double *ll_out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ngroups = (n + 31) / 32;
    // not unrolled: one group's samples in flight per warp keeps the caller's register count
#pragma unroll 1
    for (int g = warp; g < ngroups; g += nw) {
        const int j = g * 32 + lane;
        double v = j < n ? term(j) : 0.0;
        v = warp_sum_f64(v);
        if (lane == 0) s_grp[g] = v;
    }
    __syncthreads();
    const int nch = (n + kSumChunk - 1) / kSumChunk;
    for (int c = threadIdx.x; c < nch; c += blockDim.x) {
        double sum = 0.0;
        const int g1 = min(ngroups, (c + 1) * (kSumChunk / 32));
        for (int g = c * (kSumChunk / 32); g < g1; ++g) sum += s_grp[g];
        partials[first_chunk + c] = sum;
    }
    if (threadIdx.x < nch) __threadfence();  // the writers' chunk partials visible before the ticket below
    __syncthreads();
    if (warp == 0) {
        // warp 0 of the instance's last tile to finish adds the chunk partials: lane l the chunks l, l + 32,
        // ... in order, then the fixed shuffle tree
        unsigned last = 0;
        if (lane == 0) last = atomicAdd(tickets + inst, 1u) == (unsigned)tiles_of_inst - 1u;
        if (__shfl_sync(FULL, last, 0)) {
            __threadfence();
            const volatile double *p = partials + (int64_t)inst * chunks_of_inst;
            double tot = 0.0;
            for (int k = lane; k < chunks_of_inst; k += 32) tot += p[k];
            tot = warp_sum_f64(tot);
            if (lane == 0) {
                ll_out[inst] = tot;
                tickets[inst] = 0u;  // ready for the next call
            }
        }
    }
    __syncthreads();
}

}  // namespace cpab
