// cpab_mcmc.h -- launch descriptor of cpab_mcmc.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cpab {

struct McmcArgs {
    int C, d;                   // chains, parameters per chain
    double *theta;              // [C, d] current state (updated on accept)
    double *theta_prop;         // [C, d] proposal
    const double *prop_std;     // [d] proposal standard deviation per coordinate
    double scale;               // proposal scale
    double *ll;                 // [C] current log-likelihood (updated on accept)
    const double *ll_prop;      // [C] log-likelihood of the proposal
    double inv_npts;            // ratio weight (1/nPts: the average log-likelihood)
    const double *prior_prec;   // [d, d] prior precision or nullptr
    double *lp;                 // [C] current log prior (with prior_prec)
    double wlp;                 // weight of the log-prior ratio
    int rule;                   // 0: the reference's test, 1: textbook Metropolis
    uint64_t seed;
    int64_t *step;              // device step counter
    int64_t *n_accepted;        // [C] or nullptr
};

// Local (vertex-velocity) proposal tables and draws.
struct LocalProposalArgs {
    int C, d, dim, nV;
    const double *theta;        // [C, d]
    double *theta_prop;         // [C, d]
    const double *E;            // [nV, dim, d]  velocity at vertex k = E[k] theta
    const double *G;            // [nV, d, dim]  theta change for a velocity change at vertex k
    const int *bdry;            // [nV] vertex on the domain boundary
    double s;                   // step of the velocity perturbation
    uint64_t seed;
    const int64_t *step;
};

cudaError_t launch_mcmc_propose(const McmcArgs &a, cudaStream_t s);
cudaError_t launch_mcmc_propose_local(const LocalProposalArgs &a, cudaStream_t s);
cudaError_t launch_mcmc_accept(const McmcArgs &a, cudaStream_t s);
cudaError_t launch_mcmc_advance(int64_t *step, cudaStream_t s);

}  // namespace cpab
