// cpab_mcmc.cu -- batched Metropolis-Hastings over C independent chains.
//
// One step (cpab/cpaNd/inference/Metropolis.py:41-85 with the Gaussian
// random-walk proposal of cpab/cpaNd/inference/Proposal.py:29-64):
//   k_mcmc_propose   theta' = theta + scale * prop_std .* z,  z ~ N(0, I)
//   (cpab_theta_to_trels + cpab_register_ll on theta')
//   k_mcmc_accept    log_ratio = (ll' - ll) * inv_npts + wlp * (lp' - lp);
//                    accept if log_ratio > 0, else by a uniform u:
//                      rule 0 (the reference's test, Metropolis.py:77-82):
//                             accept if log(u) > log_ratio
//                      rule 1 (textbook Metropolis): accept if log(u) < log_ratio
//   k_mcmc_advance   step counter += 1
// The step index lives in device memory so that a captured CUDA graph of
// several steps can be replayed.
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011), counter (chain, step, stream, j),
// key = seed.  Two 32-bit words make one double uniform in (0, 1); normals by
// Box-Muller.  oracle/oracle.py reproduces the same stream on the CPU.
#include <math_constants.h>

#include "cpab_device.cuh"
#include "cpab_mcmc.h"

namespace cpab {

struct U4 {
    unsigned x, y, z, w;
};

__host__ __device__ __forceinline__ void mulhilo(unsigned a, unsigned b, unsigned &hi, unsigned &lo)
{
    unsigned long long p = (unsigned long long)a * (unsigned long long)b;
    hi = (unsigned)(p >> 32);
    lo = (unsigned)p;
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, unsigned k0, unsigned k1)
{
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        unsigned hi0, lo0, hi1, lo1;
        mulhilo(M0, c.x, hi0, lo0);
        mulhilo(M1, c.z, hi1, lo1);
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// (0, 1) double from two words: 53 random bits, never 0 or 1.
__device__ __forceinline__ double u53(unsigned hi, unsigned lo)
{
    unsigned long long m = ((unsigned long long)(hi >> 5) << 26) | (unsigned long long)(lo >> 6);
    return ((double)m + 0.5) * (1.0 / 9007199254740992.0);
}

enum { STREAM_PROPOSAL = 0, STREAM_ACCEPT = 1, STREAM_LOCAL = 2 };

// One thread per (chain, pair of coordinates).
__global__ void k_mcmc_propose(McmcArgs a)
{
    const int pairs = (a.d + 1) / 2;
    const int64_t step = *a.step;
    const unsigned k0 = (unsigned)a.seed, k1 = (unsigned)(a.seed >> 32);
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < (int64_t)a.C * pairs;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int chain = (int)(g / pairs), j = (int)(g - (int64_t)chain * pairs);
        U4 c{(unsigned)chain, (unsigned)step, (unsigned)(((unsigned long long)step >> 32) << 8 | STREAM_PROPOSAL),
             (unsigned)j};
        U4 r = philox4x32_10(c, k0, k1);
        double u1 = u53(r.x, r.y), u2 = u53(r.z, r.w);
        double rad = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        const int i0 = 2 * j, i1 = 2 * j + 1;
        const double *th = a.theta + (int64_t)chain * a.d;
        double *tp = a.theta_prop + (int64_t)chain * a.d;
        tp[i0] = th[i0] + a.scale * a.prop_std[i0] * (rad * cs);
        if (i1 < a.d) tp[i1] = th[i1] + a.scale * a.prop_std[i1] * (rad * sn);
    }
}

// lp(theta) = -0.5 theta^T P theta (the Gaussian log prior up to a constant,
// cpab/cpaNd/model/_ScaleDependentLogPrior.py).
__device__ double log_prior(const double *th, const double *P, int d)
{
    double s = 0.0;
    for (int i = 0; i < d; ++i) {
        double r = 0.0;
        for (int j = 0; j < d; ++j) r += P[(int64_t)i * d + j] * th[j];
        s += th[i] * r;
    }
    return -0.5 * s;
}

// One thread per chain.
__global__ void k_mcmc_accept(McmcArgs a)
{
    const int64_t step = *a.step;
    const unsigned k0 = (unsigned)a.seed, k1 = (unsigned)(a.seed >> 32);
    for (int chain = blockIdx.x * blockDim.x + threadIdx.x; chain < a.C; chain += gridDim.x * blockDim.x) {
        const double llp = a.ll_prop[chain];
        double log_ratio = (llp - a.ll[chain]) * a.inv_npts;
        double lpp = 0.0;
        const double *tp = a.theta_prop + (int64_t)chain * a.d;
        if (a.prior_prec && a.lp) {
            lpp = log_prior(tp, a.prior_prec, a.d);
            log_ratio += a.wlp * (lpp - a.lp[chain]);
        }
        bool accept;
        if (log_ratio > 0) {
            accept = true;
        } else {
            U4 c{(unsigned)chain, (unsigned)step, (unsigned)(((unsigned long long)step >> 32) << 8 | STREAM_ACCEPT),
                 0u};
            U4 r = philox4x32_10(c, k0, k1);
            double lu = log(u53(r.x, r.y));
            accept = (a.rule == 0) ? (lu > log_ratio) : (lu < log_ratio);
        }
        // NaN likelihoods never win: a proposal whose ratio is NaN is rejected
        if (log_ratio != log_ratio) accept = false;
        if (accept) {
            double *th = a.theta + (int64_t)chain * a.d;
            for (int i = 0; i < a.d; ++i) th[i] = tp[i];
            a.ll[chain] = llp;
            if (a.prior_prec && a.lp) a.lp[chain] = lpp;
            if (a.n_accepted) a.n_accepted[chain] += 1;
        }
    }
}

// Local proposal (cpab/cpaNd/inference/Proposal.py:65-130): pick a vertex k
// uniformly, add s * z (z ~ N(0, I_dim)) to its velocity -- or, for a vertex
// on the domain boundary, set its velocity to 0 -- and map the change to
// theta: theta' = theta + G[k] dv.  One warp per chain; Philox stream 2,
// word 0 of counter (chain, step, 2, 0) picks k, counters (.., 1 + p) give the
// normal pairs.
__global__ void k_mcmc_propose_local(LocalProposalArgs a)
{
    const int lane = threadIdx.x & 31;
    const int64_t step = *a.step;
    const unsigned k0 = (unsigned)a.seed, k1 = (unsigned)(a.seed >> 32);
    const unsigned hi = (unsigned)(((unsigned long long)step >> 32) << 8 | STREAM_LOCAL);
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int chain = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; chain < a.C; chain += nwarps) {
        const U4 r0 = philox4x32_10(U4{(unsigned)chain, (unsigned)step, hi, 0u}, k0, k1);
        int k = (int)(u53(r0.x, r0.y) * (double)a.nV);
        k = k < a.nV ? k : a.nV - 1;
        const double *th = a.theta + (int64_t)chain * a.d;
        double dv[3] = {0.0, 0.0, 0.0};
        if (a.bdry[k]) {
            // dv = -v_k = -E[k] theta (lanes split the dot products, fixed-order warp sum)
            for (int r = 0; r < a.dim; ++r) {
                const double *e = a.E + ((int64_t)k * a.dim + r) * a.d;
                double acc = 0.0;
                for (int i = lane; i < a.d; i += 32) acc += e[i] * th[i];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
                dv[r] = -acc;
            }
        } else {
            for (int p = 0; 2 * p < a.dim; ++p) {
                const U4 r = philox4x32_10(U4{(unsigned)chain, (unsigned)step, hi, 1u + (unsigned)p}, k0, k1);
                const double u1 = u53(r.x, r.y), u2 = u53(r.z, r.w);
                const double rad = sqrt(-2.0 * log(u1));
                double sn, cs;
                sincospi(2.0 * u2, &sn, &cs);
                dv[2 * p] = a.s * rad * cs;
                if (2 * p + 1 < a.dim) dv[2 * p + 1] = a.s * rad * sn;
            }
        }
        double *tp = a.theta_prop + (int64_t)chain * a.d;
        const double *g = a.G + (int64_t)k * a.d * a.dim;
        for (int i = lane; i < a.d; i += 32) {
            double v = th[i];
            for (int r = 0; r < a.dim; ++r) v += g[(int64_t)i * a.dim + r] * dv[r];
            tp[i] = v;
        }
    }
}

__global__ void k_mcmc_advance(int64_t *step) { *step += 1; }

cudaError_t launch_mcmc_propose(const McmcArgs &a, cudaStream_t s)
{
    const int64_t n = (int64_t)a.C * ((a.d + 1) / 2);
    int grid = (int)((n + 255) / 256);
    if (grid < 1) grid = 1;
    k_mcmc_propose<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_mcmc_propose_local(const LocalProposalArgs &a, cudaStream_t s)
{
    int grid = (a.C * 32 + 255) / 256;
    if (grid < 1) grid = 1;
    k_mcmc_propose_local<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_mcmc_accept(const McmcArgs &a, cudaStream_t s)
{
    int grid = (a.C + 127) / 128;
    if (grid < 1) grid = 1;
    k_mcmc_accept<<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_mcmc_advance(int64_t *step, cudaStream_t s)
{
    k_mcmc_advance<<<1, 1, 0, s>>>(step);
    return cudaGetLastError();
}

}  // namespace cpab
