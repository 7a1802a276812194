// cpab_grad.cu -- adjoint (reverse-mode) gradient of the midpoint scheme.
//
// Forward (calc_T_simple, cpab/gpu/calc_2Dto2D.cu:412-445): nTimeSteps *
// nStepsODE explicit-midpoint sub-steps, each with the matrix of the cell
// that holds the sub-step's start point,
//     v = L p + t,  pm = p + h/2 v,  v2 = L pm + t,  p' = p + h v2.
// The reference's own sensitivity code (solveODE2 / calc_grad_theta,
// calc_2Dto2D.cu:202-319,448-491; never bound, cpab/gpu/Calcs.py:196) carries
// dp/dtheta forward for every basis vector.  Here the gradient of a scalar
// loss runs backwards instead: given g = dLoss/dT(x) per point,
//     a = h g',  dL += a pm^T, dt += a,  dpm = L^T a,
//     b = h/2 dpm,  dL += b p^T, dt += b,  g = g' + dpm + L^T b,
// summed per cell into dLoss/dA [nC, D, D+1]; dLoss/dtheta = B^T dLoss/dA
// (k_bt_times).  This is the exact gradient of the discrete forward map.
//
// Memory: positions at the start of every `ck`-th time step are kept in
// scratch ([ceil(nT/ck), nPts, D] float64); the start of any other step is
// recomputed from the previous checkpoint (ck = 1 stores all, ck = nT only
// the input).  Inside a time step the sub-steps are replayed in groups of
// kGroup from kGroup start points held in a small per-thread buffer.
#include "cpab_integrate.cuh"
#include "cpab_grad.h"
#include "cpab_launch.h"

namespace cpab {

constexpr int kGroup = 16;   // sub-steps per replay group; nStepsODE <= kGroup * kGroup

template <int DIM, int TESS>
__device__ __forceinline__ void substeps(const Tess &t, const double *sA, double *p, double h, int n)
{
    constexpr int NE = DIM * (DIM + 1);
    for (int k = 0; k < n; ++k) {
        int c = exact_cell<DIM, TESS>(t, p);
        exact_midpoint<DIM>(p, sA + c * NE, h);
    }
}

template <int DIM, int TESS>
__global__ void __launch_bounds__(128) k_grad_simple(GradArgs a)
{
    constexpr int NE = DIM * (DIM + 1), NH = DIM + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sA = reinterpret_cast<double *>(smem_raw);
    double *sG = sA + a.t.nC * NE;
    const int inst = blockIdx.y;
    const int tab = a.t.nC * NE;
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        sA[i] = a.A[(size_t)inst * tab + i];
        sG[i] = 0.0;
    }
    __syncthreads();
    const double h = XDIV(a.dt, (double)a.nStepsODE);
    const int nT = a.nTimeSteps, nODE = a.nStepsODE, ck = a.ck;
    const int ngroups = (nODE + kGroup - 1) / kGroup;
    const int64_t n = a.n_per_inst;
    const int64_t total = n * a.N;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t gi = (int64_t)inst * n + j;
        double p[DIM];
        load_pt<DIM, double>(a.pts, gi, p);
        // forward with checkpoints
        for (int s = 0; s < nT; ++s) {
            if (s % ck == 0) store_pt<DIM, double>(a.ckpt, (int64_t)(s / ck) * total + gi, p);
            substeps<DIM, TESS>(a.t, sA, p, h, nODE);
        }
        if (a.out) store_pt<DIM, double>(a.out, gi, p);
        double g[DIM];
        load_pt<DIM, double>(a.grad_out, gi, g);
        double acc[NE];
#pragma unroll
        for (int e = 0; e < NE; ++e) acc[e] = 0.0;
        int acc_cell = -1;
        double buf1[kGroup][DIM], buf2[kGroup][DIM];
        for (int s = nT - 1; s >= 0; --s) {
            // start of time step s
            double q[DIM];
            load_pt<DIM, double>(a.ckpt, (int64_t)(s / ck) * total + gi, q);
            substeps<DIM, TESS>(a.t, sA, q, h, s % ck * nODE);
            // group starts
            for (int k = 0; k < nODE; ++k) {
                if (k % kGroup == 0) {
#pragma unroll
                    for (int i = 0; i < DIM; ++i) buf1[k / kGroup][i] = q[i];
                }
                int c = exact_cell<DIM, TESS>(a.t, q);
                exact_midpoint<DIM>(q, sA + c * NE, h);
            }
            for (int gr = ngroups - 1; gr >= 0; --gr) {
                const int k0 = gr * kGroup, k1 = min(nODE, k0 + kGroup);
                double r[DIM];
#pragma unroll
                for (int i = 0; i < DIM; ++i) r[i] = buf1[gr][i];
                for (int k = k0; k < k1; ++k) {
#pragma unroll
                    for (int i = 0; i < DIM; ++i) buf2[k - k0][i] = r[i];
                    int c = exact_cell<DIM, TESS>(a.t, r);
                    exact_midpoint<DIM>(r, sA + c * NE, h);
                }
                for (int k = k1 - 1; k >= k0; --k) {
                    double pk[DIM];
#pragma unroll
                    for (int i = 0; i < DIM; ++i) pk[i] = buf2[k - k0][i];
                    const int c = exact_cell<DIM, TESS>(a.t, pk);
                    const double *M = sA + c * NE;
                    if (c != acc_cell) {
                        if (acc_cell >= 0) {
#pragma unroll
                            for (int e = 0; e < NE; ++e) {
                                atomicAdd(sG + acc_cell * NE + e, acc[e]);
                                acc[e] = 0.0;
                            }
                        }
                        acc_cell = c;
                    }
                    // recompute v and pm of the forward sub-step
                    double v[DIM], pm[DIM];
                    exact_affine<DIM>(v, M, pk);
#pragma unroll
                    for (int i = 0; i < DIM; ++i) pm[i] = pk[i] + h * v[i] / 2.;
                    double av[DIM], dpm[DIM], b[DIM];
#pragma unroll
                    for (int i = 0; i < DIM; ++i) av[i] = h * g[i];
#pragma unroll
                    for (int jj = 0; jj < DIM; ++jj) {
                        double s2 = 0.0;
#pragma unroll
                        for (int i = 0; i < DIM; ++i) s2 += M[i * NH + jj] * av[i];
                        dpm[jj] = s2;
                    }
#pragma unroll
                    for (int i = 0; i < DIM; ++i) b[i] = 0.5 * h * dpm[i];
#pragma unroll
                    for (int i = 0; i < DIM; ++i) {
#pragma unroll
                        for (int jj = 0; jj < DIM; ++jj) acc[i * NH + jj] += av[i] * pm[jj] + b[i] * pk[jj];
                        acc[i * NH + DIM] += av[i] + b[i];
                    }
#pragma unroll
                    for (int jj = 0; jj < DIM; ++jj) {
                        double s2 = 0.0;
#pragma unroll
                        for (int i = 0; i < DIM; ++i) s2 += M[i * NH + jj] * b[i];
                        g[jj] += dpm[jj] + s2;
                    }
                }
            }
        }
        if (acc_cell >= 0) {
#pragma unroll
            for (int e = 0; e < NE; ++e) atomicAdd(sG + acc_cell * NE + e, acc[e]);
        }
        if (a.grad_in) store_pt<DIM, double>(a.grad_in, gi, g);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        double v = sG[i];
        if (v != 0.0) atomicAdd(a.gA + (size_t)inst * tab + i, v);
    }
}

// out[n, j] = scale * sum_k B[k, j] * G[n, k]  (dLoss/dtheta = B^T dLoss/dA)
__global__ void k_bt_times(const double *B, const double *G, double *out, int DA, int d, int N, double scale)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < (int64_t)N * d;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int n = (int)(g / d), j = (int)(g - (int64_t)n * d);
        const double *Gn = G + (int64_t)n * DA;
        double s = 0.0;
        for (int k = 0; k < DA; ++k) s = fma(B[(int64_t)k * d + j], Gn[k], s);
        out[g] = scale * s;
    }
}

template <int DIM, int TESS>
static cudaError_t launch_grad_t(const GradArgs &a, cudaStream_t s)
{
    constexpr int NE = DIM * (DIM + 1);
    size_t smem = (size_t)2 * a.t.nC * NE * sizeof(double);
    auto kern = k_grad_simple<DIM, TESS>;
    if (smem > kSmemOptInAbove) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int64_t bx = (a.n_per_inst + 127) / 128;
    int64_t cap = (int64_t)num_sms() * 8 / (a.N > 0 ? a.N : 1) + 1;
    if (bx > cap) bx = cap;
    if (bx < 1) bx = 1;
    dim3 grid((unsigned)bx, (unsigned)a.N);
    kern<<<grid, 128, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_grad_simple(const GradArgs &a, cudaStream_t s)
{
    const int dim = a.t.dim, tess = a.t.tess;
    if (dim == 1) return launch_grad_t<1, 2>(a, s);
    if (dim == 2) return tess == 1 ? launch_grad_t<2, 1>(a, s) : launch_grad_t<2, 2>(a, s);
    return tess == 1 ? launch_grad_t<3, 1>(a, s) : launch_grad_t<3, 2>(a, s);
}

cudaError_t launch_bt_times(const double *B, const double *G, double *out, int DA, int d, int N, double scale,
                            cudaStream_t s)
{
    int64_t n = (int64_t)N * d;
    int grid = (int)((n + 127) / 128);
    if (grid < 1) grid = 1;
    if (grid > num_sms() * 16) grid = num_sms() * 16;
    k_bt_times<<<grid, 128, 0, s>>>(B, G, out, DA, d, N, scale);
    return cudaGetLastError();
}

}  // namespace cpab
