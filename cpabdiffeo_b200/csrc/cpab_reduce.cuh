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

}  // namespace cpab
