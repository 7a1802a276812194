// cpab_launch.h -- host-side launchers of cpab_kernels.cu / cpab_remap.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cpab_internal.h"

namespace cpab {

// Launch shape of the integration kernel (chosen by the autotuner).
struct LaunchCfg {
    int block = 256;       // threads per CTA (multiple of 32, <= 256)
    int ctas_per_sm = 32;  // cap on resident CTAs per SM of the persistent grid (occupancy decides below it)
    int grid = 0;          // explicit grid (0 = persistent default)
    int tile_pts = 2048;   // points per CTA tile
    int sort = 0;          // cell-sort the points of each tile
    int max_ctas = 0;      // cap on the CTAs of every persistent launch of the context (0 = none)
};

// Kernels opt in to more than the default 48 KB of shared memory when their
// dynamic size exceeds this (their static shared memory comes on top).
constexpr size_t kSmemOptInAbove = 40 * 1024;

int num_sms();

// Points per tile of a uniform integration launch over `total` points: the
// configured tile, or a smaller one (a multiple of 32, at least 64) when the
// launch has too few points to give every SM four tiles -- one transform of a
// few hundred thousand points would otherwise occupy fewer SMs than the GPU
// has.  Per-point results do not depend on the tiling.  (The likelihood
// kernels keep the configured tile: their sums follow the tiles, and a tile
// that depended on the batch would break "the same alone and in a batch".)
inline int small_launch_tile(int64_t total, int tile_pts)
{
    const int64_t want = 4 * (int64_t)num_sms();
    if (total >= want * tile_pts) return tile_pts;
    int64_t t = (total + want - 1) / want;
    t = (t + 31) / 32 * 32;
    if (t < 64) t = 64;
    return (int)(t < tile_pts ? t : tile_pts);
}
int persistent_grid_impl(const void *kern, const LaunchCfg &cfg, size_t smem);
template <typename K>
inline int persistent_grid(K kern, const LaunchCfg &cfg, size_t smem)
{
    return persistent_grid_impl(reinterpret_cast<const void *>(kern), cfg, smem);
}

cudaError_t launch_integrate(const IntegrateArgs &a, int prec, int scheme, const LaunchCfg &cfg, cudaStream_t s);
cudaError_t launch_integrate_exact1d(const IntegrateArgs &a, int prec, const LaunchCfg &cfg, cudaStream_t s);
size_t exact1d_smem_bytes(int nC, int tile_pts, int sort, int prec);
cudaError_t launch_tile_prefix(const int64_t *offsets, int64_t *prefix, int N, int tile_pts, cudaStream_t s);
cudaError_t launch_trajectory(const IntegrateArgs &a, int64_t nPts, cudaStream_t s);
cudaError_t launch_cell_idx(const Tess &t, const double *pts, int32_t *out, int64_t n, cudaStream_t s);
cudaError_t launch_calc_v(const Tess &t, const double *A, const double *pts, double *out, int64_t n, cudaStream_t s);
cudaError_t launch_expm(int dim, const double *A, double *signedA, double *T, int64_t n_cells, double dt,
                        double sign, cudaStream_t s);
cudaError_t launch_theta_to_trels(int dim, const double *B, const double *theta, int d, int nC, int N, double dt,
                                  double sign, double *A, double *signedA, double *T, cudaStream_t s);

}  // namespace cpab
