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
// the input).  Inside a time step the sub-steps are replayed once, keeping
// every sub-step's start point and cell in a per-thread array.
//
// k_grad_ref: the same for the reference scheme (calc_T, calc_2Dto2D.cu:
// 348-408): a time step is either the closed-form step q = T_c [p; 1] with
// T_c = expm(dt A_c), kept when q stays in cell c, or nStepsODE sub-steps as
// above.  Backwards through a kept step
//     dT_c += g [p; 1]^T,   g = T_lin^T g,
// and through a fallback step the sub-step adjoint.  The per-cell sums dT_c
// become dLoss/dA_c once per instance and cell (k_frechet_adjoint):
//     dA_c += dt L(X^T, dT_c),  X = dt [A_c; 0],
// L the Frechet derivative of expm, read off the top-right block of
// expm([[X^T, G], [0, X^T]]).  This is the exact gradient of the discrete
// map along the branch the forward took (kept / fallback, cells); where a
// step changes branch the map itself is discontinuous.
#include "cpab_integrate.cuh"
#include "cpab_grad.h"
#include "cpab_launch.h"

namespace cpab {

constexpr int kMaxSubsteps = 256;  // sub-steps per time step the adjoint keeps (cpab_grad_theta* check)

template <int DIM, int TESS>
__device__ __forceinline__ void substeps(const Tess &t, const double *sA, double *p, double h, int n)
{
    constexpr int NE = DIM * (DIM + 1);
    for (int k = 0; k < n; ++k) {
        int c = exact_cell<DIM, TESS>(t, p);
        exact_midpoint<DIM>(p, sA + c * NE, h);
    }
}

// Per-thread accumulator of one cell's dLoss/d(matrix) entries, added to the
// CTA's shared sums when the cell changes (c = -1: flush).
template <int NE>
__device__ __forceinline__ void acc_switch(double *sG, double *acc, int &acc_cell, int c)
{
    if (c == acc_cell) return;
    if (acc_cell >= 0) {
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            atomicAdd(sG + acc_cell * NE + e, acc[e]);
            acc[e] = 0.0;
        }
    }
    acc_cell = c;
}

// Backwards through the nODE sub-steps of one time step that starts at q
// (q is consumed): g = dLoss/d(end of the step) on entry, dLoss/d(start) on
// return; dLoss/dA of the cells used is accumulated (acc / acc_cell / sG).
// One forward pass keeps every sub-step's start point and cell in a
// per-thread array (nODE <= 256: at most 7 KB of local memory), then the
// adjoint runs down it.
template <int DIM, int TESS>
__device__ __forceinline__ void adjoint_substeps(const Tess &t, const double *sA, double *sG, double *q, double *g,
                                                 double h, int nODE, double *acc, int &acc_cell)
{
    constexpr int NE = DIM * (DIM + 1), NH = DIM + 1;
    double xs[kMaxSubsteps][DIM];
    int cs[kMaxSubsteps];
    for (int k = 0; k < nODE; ++k) {
        const int c = exact_cell<DIM, TESS>(t, q);
#pragma unroll
        for (int i = 0; i < DIM; ++i) xs[k][i] = q[i];
        cs[k] = c;
        exact_midpoint<DIM>(q, sA + c * NE, h);
    }
    for (int k = nODE - 1; k >= 0; --k) {
        double pk[DIM];
#pragma unroll
        for (int i = 0; i < DIM; ++i) pk[i] = xs[k][i];
        const int c = cs[k];
        const double *M = sA + c * NE;
        acc_switch<NE>(sG, acc, acc_cell, c);
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

template <int DIM, int TESS>
__global__ void __launch_bounds__(128) k_grad_simple(GradArgs a)
{
    constexpr int NE = DIM * (DIM + 1);
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
        for (int s = nT - 1; s >= 0; --s) {
            // start of time step s
            double q[DIM];
            load_pt<DIM, double>(a.ckpt, (int64_t)(s / ck) * total + gi, q);
            substeps<DIM, TESS>(a.t, sA, q, h, s % ck * nODE);
            adjoint_substeps<DIM, TESS>(a.t, sA, sG, q, g, h, nODE, acc, acc_cell);
        }
        acc_switch<NE>(sG, acc, acc_cell, -1);
        if (a.grad_in) store_pt<DIM, double>(a.grad_in, gi, g);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        double v = sG[i];
        if (v != 0.0) atomicAdd(a.gA + (size_t)inst * tab + i, v);
    }
}

// One time step of the reference scheme from p (calc_T, the FP64 arithmetic
// of k_integrate): the closed-form step when its end point stays in the
// cell, else nODE sub-steps.  Returns whether the closed-form step was kept.
template <int DIM, int TESS>
__device__ __forceinline__ bool ref_step(const Tess &t, const double *sA, const double *sT, double *p, double h,
                                         int nODE)
{
    constexpr int NE = DIM * (DIM + 1);
    const int c = exact_cell<DIM, TESS>(t, p);
    double q[DIM];
    exact_affine<DIM>(q, sT + c * NE, p);
    if (exact_cell<DIM, TESS>(t, q) == c) {
#pragma unroll
        for (int i = 0; i < DIM; ++i) p[i] = q[i];
        return true;
    }
    substeps<DIM, TESS>(t, sA, p, h, nODE);
    return false;
}

// SACC: the gradient sums in shared memory, added to gA / gT at the end;
// else (large tables) the per-thread accumulators go straight to gA / gT, so
// that shared memory holds the tables only and more CTAs fit on an SM.
template <int DIM, int TESS, bool SACC>
__global__ void __launch_bounds__(128) k_grad_ref(GradArgs a)
{
    constexpr int NE = DIM * (DIM + 1), NH = DIM + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tab = a.t.nC * NE;
    const int inst = blockIdx.y;
    double *sA = reinterpret_cast<double *>(smem_raw);
    double *sT = sA + tab;
    double *sGA = SACC ? sT + tab : a.gA + (size_t)inst * tab;   // dLoss/dA from sub-steps
    double *sGT = SACC ? sGA + tab : a.gT + (size_t)inst * tab;  // dLoss/dT from closed-form steps
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        sA[i] = a.A[(size_t)inst * tab + i];
        sT[i] = a.T[(size_t)inst * tab + i];
        if (SACC) {
            sGA[i] = 0.0;
            sGT[i] = 0.0;
        }
    }
    __syncthreads();
    const double h = XDIV(a.dt, (double)a.nStepsODE);
    const int nT = a.nTimeSteps, nODE = a.nStepsODE, ck = a.ck;
    const int64_t n = a.n_per_inst;
    const int64_t total = n * a.N;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t gi = (int64_t)inst * n + j;
        double p[DIM];
        load_pt<DIM, double>(a.pts, gi, p);
        for (int s = 0; s < nT; ++s) {
            if (s % ck == 0) store_pt<DIM, double>(a.ckpt, (int64_t)(s / ck) * total + gi, p);
            ref_step<DIM, TESS>(a.t, sA, sT, p, h, nODE);
        }
        if (a.out) store_pt<DIM, double>(a.out, gi, p);
        double g[DIM];
        load_pt<DIM, double>(a.grad_out, gi, g);
        double accA[NE], accT[NE];
#pragma unroll
        for (int e = 0; e < NE; ++e) accA[e] = accT[e] = 0.0;
        int cellA = -1, cellT = -1;
        for (int s = nT - 1; s >= 0; --s) {
            double q[DIM];
            load_pt<DIM, double>(a.ckpt, (int64_t)(s / ck) * total + gi, q);
            for (int r = 0; r < s % ck; ++r) ref_step<DIM, TESS>(a.t, sA, sT, q, h, nODE);
            // time step s from q, along the forward's branch
            const int c = exact_cell<DIM, TESS>(a.t, q);
            const double *T = sT + c * NE;
            double y[DIM];
            exact_affine<DIM>(y, T, q);
            if (exact_cell<DIM, TESS>(a.t, y) == c) {
                acc_switch<NE>(sGT, accT, cellT, c);
#pragma unroll
                for (int i = 0; i < DIM; ++i) {
#pragma unroll
                    for (int k = 0; k < DIM; ++k) accT[i * NH + k] += g[i] * q[k];
                    accT[i * NH + DIM] += g[i];
                }
                double gn[DIM];
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    double s2 = 0.0;
#pragma unroll
                    for (int i = 0; i < DIM; ++i) s2 += T[i * NH + k] * g[i];
                    gn[k] = s2;
                }
#pragma unroll
                for (int k = 0; k < DIM; ++k) g[k] = gn[k];
            } else {
                adjoint_substeps<DIM, TESS>(a.t, sA, sGA, q, g, h, nODE, accA, cellA);
            }
        }
        acc_switch<NE>(sGA, accA, cellA, -1);
        acc_switch<NE>(sGT, accT, cellT, -1);
        if (a.grad_in) store_pt<DIM, double>(a.grad_in, gi, g);
    }
    if (!SACC) return;
    __syncthreads();
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        const double va = sGA[i], vt = sGT[i];
        if (va != 0.0) atomicAdd(a.gA + (size_t)inst * tab + i, va);
        if (vt != 0.0) atomicAdd(a.gT + (size_t)inst * tab + i, vt);
    }
}

// E = expm(Z) for a small K x K matrix: scaling and squaring (Moler & Van
// Loan, "Nineteen dubious ways to compute the exponential of a matrix",
// method 3) with the degree-18 Taylor polynomial of Z / 2^s,
// ||Z / 2^s||_1 <= 1/2 (truncation below 1e-22 relative).  Z is scaled in
// place.
template <int K>
__device__ void expm_small(double (&Z)[K][K], double (&E)[K][K])
{
    double nrm = 0.0;
    for (int j = 0; j < K; ++j) {
        double cs = 0.0;
        for (int i = 0; i < K; ++i) cs += fabs(Z[i][j]);
        nrm = fmax(nrm, cs);
    }
    int sq = 0;
    while (nrm > 0.5 && sq < 60) {
        nrm *= 0.5;
        ++sq;
    }
    const double sc = ldexp(1.0, -sq);
    double Tm[K][K], W[K][K];
    for (int i = 0; i < K; ++i)
        for (int j = 0; j < K; ++j) {
            Z[i][j] *= sc;
            Tm[i][j] = E[i][j] = (i == j) ? 1.0 : 0.0;
        }
    for (int k = 1; k <= 18; ++k) {
        const double inv = 1.0 / (double)k;
        for (int i = 0; i < K; ++i)
            for (int j = 0; j < K; ++j) {
                double s2 = 0.0;
                for (int m = 0; m < K; ++m) s2 += Tm[i][m] * Z[m][j];
                W[i][j] = s2 * inv;
            }
        for (int i = 0; i < K; ++i)
            for (int j = 0; j < K; ++j) {
                Tm[i][j] = W[i][j];
                E[i][j] += W[i][j];
            }
    }
    for (int r = 0; r < sq; ++r) {
        for (int i = 0; i < K; ++i)
            for (int j = 0; j < K; ++j) {
                double s2 = 0.0;
                for (int m = 0; m < K; ++m) s2 += E[i][m] * E[m][j];
                W[i][j] = s2;
            }
        for (int i = 0; i < K; ++i)
            for (int j = 0; j < K; ++j) E[i][j] = W[i][j];
    }
}

// gA[c] += dt L(X^T, G_c) for every (instance, cell) c, X = dt [A_c; 0]
// (homogeneous, last row zero) and G_c = [gT_c; 0].  L is linear in G, so G
// is scaled to max |entry| 1 before the exponential and the block scaled
// back, which keeps the squaring count set by X.
template <int DIM>
__global__ void k_frechet_adjoint(const double *A, const double *gT, double *gA, int total, double dt)
{
    constexpr int M = DIM + 1, K = 2 * M, NE = DIM * M;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
        const double *a = A + (size_t)idx * NE;
        const double *g = gT + (size_t)idx * NE;
        double gs = 0.0;
        for (int e = 0; e < NE; ++e) gs = fmax(gs, fabs(g[e]));
        if (!(gs > 0.0)) continue;  // no closed-form step in this cell
        double Z[K][K], E[K][K];
        for (int i = 0; i < K; ++i)
            for (int j = 0; j < K; ++j) Z[i][j] = 0.0;
        for (int i = 0; i < DIM; ++i)
            for (int j = 0; j < M; ++j) {
                const double x = dt * a[i * M + j];  // X[i][j]
                Z[j][i] = x;                         // X^T, top left
                Z[M + j][M + i] = x;                 // X^T, bottom right
                Z[i][M + j] = g[i * M + j] / gs;     // G, top right
            }
        expm_small<K>(Z, E);
        for (int i = 0; i < DIM; ++i)
            for (int j = 0; j < M; ++j) gA[(size_t)idx * NE + i * M + j] += dt * gs * E[i][M + j];
    }
}

// ------------------------------------------------------------ FP32 adjoint of calc_T
//
// The FP32 forward (k_integrate<float>, SCHEME_REF) keeps each coordinate as
// a compensated pair hi + lo and moves it by x + M[x; 1] with the cell's
// float T - I (closed-form step) or S - I (one midpoint sub-step, S the
// sub-step's affine map).  k_grad_ref_f32 replays exactly that arithmetic
// (checkpoints hold hi and lo) and goes backwards through
//     x' = x + M_c [x; 1]:   dM_c += g [x; 1]^T,  g = g + M_lin^T g,
// with dM summed per cell for T (gT) and for S (gS).  Per instance and cell,
// dLoss/dA then follows in FP64 from gT through the expm Frechet adjoint and
// from gS through the derivative of S - I = [hL + h^2/2 L^2 | hb + h^2/2 Lb]
// (k_substep_map_adjoint).

template <int NE>
__device__ __forceinline__ void acc_switch_f(double *sG, float *acc, int &acc_cell, int c)
{
    if (c == acc_cell) return;
    if (acc_cell >= 0) {
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            atomicAdd(sG + acc_cell * NE + e, (double)acc[e]);
            acc[e] = 0.0f;
        }
    }
    acc_cell = c;
}

// x' = x + M[x; 1] on the compensated state (the float advance() of the lane scheduler)
template <int DIM>
__device__ __forceinline__ void f32_map(PState<DIM, float> &st, const float *M)
{
    constexpr int NE = DIM * (DIM + 1);
    float m[NE], d[DIM];
    load_cell<DIM>(M, m);
    cm_affine<DIM>(d, m, st.x);
#pragma unroll
    for (int r = 0; r < DIM; ++r) st.add(r, d[r]);
}

// One time step of calc_T in FP32 from st; returns whether the closed-form step was kept.
template <int DIM, int TESS>
__device__ __forceinline__ bool ref_step_f32(const Tess &t, const float *sS, const float *sT, PState<DIM, float> &st,
                                             int nODE)
{
    constexpr int NE = DIM * (DIM + 1);
    const int c = fast_cell<DIM, TESS>(t, st.x);
    PState<DIM, float> q = st;
    f32_map<DIM>(q, sT + c * NE);
    if (fast_cell<DIM, TESS>(t, q.x) == c) {
        st = q;
        return true;
    }
    for (int k = 0; k < nODE; ++k) f32_map<DIM>(st, sS + fast_cell<DIM, TESS>(t, st.x) * NE);
    return false;
}

// Backwards through x' = x + M[x; 1] (M column-major float, cell c): accumulate
// g [x; 1]^T into acc (row-major, as the FP64 tables) and set g += M_lin^T g.
template <int DIM>
__device__ __forceinline__ void f32_map_adjoint(const float *M, const float *x, float *g, float *acc)
{
    constexpr int NE = DIM * (DIM + 1), NH = DIM + 1;
    float m[NE];
    load_cell<DIM>(M, m);
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) acc[r * NH + k] = fmaf(g[r], x[k], acc[r * NH + k]);
        acc[r * NH + DIM] += g[r];
    }
    float gn[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        float s2 = g[k];
#pragma unroll
        for (int r = 0; r < DIM; ++r) s2 = fmaf(m[k * DIM + r], g[r], s2);
        gn[k] = s2;
    }
#pragma unroll
    for (int k = 0; k < DIM; ++k) g[k] = gn[k];
}

// Backwards through the nODE sub-steps of a fallback step starting at st
// (consumed): one forward pass keeps every sub-step's point and cell in a
// per-thread array (nODE <= 256, at most 4 KB of local memory, touched only
// by fallback steps), then the adjoint runs down it.
template <int DIM, int TESS>
__device__ __forceinline__ void adjoint_substeps_f32(const Tess &t, const float *sS, double *sGS,
                                                     PState<DIM, float> &st, float *g, int nODE, float *acc,
                                                     int &acc_cell)
{
    constexpr int NE = DIM * (DIM + 1);
    float xs[kMaxSubsteps][DIM];
    int cs[kMaxSubsteps];
    for (int k = 0; k < nODE; ++k) {
        const int c = fast_cell<DIM, TESS>(t, st.x);
#pragma unroll
        for (int i = 0; i < DIM; ++i) xs[k][i] = st.x[i];
        cs[k] = c;
        f32_map<DIM>(st, sS + c * NE);
    }
    for (int k = nODE - 1; k >= 0; --k) {
        const int c = cs[k];
        acc_switch_f<NE>(sGS, acc, acc_cell, c);
        f32_map_adjoint<DIM>(sS + c * NE, xs[k], g, acc);
    }
}

template <int DIM, int TESS, bool SACC>
__global__ void __launch_bounds__(128) k_grad_ref_f32(GradArgs a)
{
    constexpr int NE = DIM * (DIM + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tab = a.t.nC * NE;
    const int inst = blockIdx.y;
    double *sums = reinterpret_cast<double *>(smem_raw);
    double *sGS = SACC ? sums : a.gS + (size_t)inst * tab;        // dLoss/dS (sub-steps)
    double *sGT = SACC ? sums + tab : a.gT + (size_t)inst * tab;  // dLoss/dT (closed-form steps)
    float *sS = reinterpret_cast<float *>(sums + (SACC ? 2 * tab : 0));
    float *sT = sS + tab;
    stage_tables<DIM, float>(a.A + (size_t)inst * tab, a.T + (size_t)inst * tab, a.t.nC, true, a.h_sub, sS, sT);
    if (SACC)
        for (int i = threadIdx.x; i < 2 * tab; i += blockDim.x) sums[i] = 0.0;
    __syncthreads();
    const int nT = a.nTimeSteps, nODE = a.nStepsODE, ck = a.ck;
    const int64_t n = a.n_per_inst;
    const int64_t total = n * a.N;
    float *ckpt = reinterpret_cast<float *>(a.ckpt);  // [ceil(nT/ck), N*n, 2*DIM]: hi, lo
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t gi = (int64_t)inst * n + j;
        float p[DIM];
        load_pt<DIM, float>(a.pts, gi, p);
        PState<DIM, float> st;
        st.set(p);
        for (int s = 0; s < nT; ++s) {
            if (s % ck == 0) {
                float *c = ckpt + ((int64_t)(s / ck) * total + gi) * 2 * DIM;
#pragma unroll
                for (int i = 0; i < DIM; ++i) {
                    c[i] = st.hi[i];
                    c[DIM + i] = st.lo[i];
                }
            }
            ref_step_f32<DIM, TESS>(a.t, sS, sT, st, nODE);
        }
        if (a.out) {
            st.get(p);
            store_pt<DIM, float>(a.out, gi, p);
        }
        float g[DIM];
        load_pt<DIM, float>(a.grad_out, gi, g);
        float accS[NE], accT[NE];
#pragma unroll
        for (int e = 0; e < NE; ++e) accS[e] = accT[e] = 0.0f;
        int cellS = -1, cellT = -1;
        for (int s = nT - 1; s >= 0; --s) {
            PState<DIM, float> q;
            const float *c = ckpt + ((int64_t)(s / ck) * total + gi) * 2 * DIM;
#pragma unroll
            for (int i = 0; i < DIM; ++i) {
                q.hi[i] = c[i];
                q.lo[i] = c[DIM + i];
                q.x[i] = q.hi[i] + q.lo[i];
            }
            for (int r = 0; r < s % ck; ++r) ref_step_f32<DIM, TESS>(a.t, sS, sT, q, nODE);
            // time step s from q, along the forward's branch
            const int cc = fast_cell<DIM, TESS>(a.t, q.x);
            PState<DIM, float> y = q;
            f32_map<DIM>(y, sT + cc * NE);
            if (fast_cell<DIM, TESS>(a.t, y.x) == cc) {
                acc_switch_f<NE>(sGT, accT, cellT, cc);
                f32_map_adjoint<DIM>(sT + cc * NE, q.x, g, accT);
            } else {
                adjoint_substeps_f32<DIM, TESS>(a.t, sS, sGS, q, g, nODE, accS, cellS);
            }
        }
        acc_switch_f<NE>(sGS, accS, cellS, -1);
        acc_switch_f<NE>(sGT, accT, cellT, -1);
        if (a.grad_in) store_pt<DIM, float>(a.grad_in, gi, g);
    }
    if (!SACC) return;
    __syncthreads();
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        const double vs = sGS[i], vt = sGT[i];
        if (vs != 0.0) atomicAdd(a.gS + (size_t)inst * tab + i, vs);
        if (vt != 0.0) atomicAdd(a.gT + (size_t)inst * tab + i, vt);
    }
}

// gA[c] += dLoss/dA through S - I = [hL + h^2/2 L^2 | hb + h^2/2 Lb] (A = [L | b]):
//     dL = h G + h^2/2 (G L^T + L^T G + g b^T),   db = h g + h^2/2 L^T g,
// G, g the linear and offset parts of gS[c].
template <int DIM>
__global__ void k_substep_map_adjoint(const double *A, const double *gS, double *gA, int total, double h)
{
    constexpr int M = DIM + 1, NE = DIM * M;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
        const double *a = A + (size_t)idx * NE;
        const double *G = gS + (size_t)idx * NE;
        double *o = gA + (size_t)idx * NE;
        const double hh = 0.5 * h * h;
        for (int i = 0; i < DIM; ++i) {
            for (int j = 0; j < DIM; ++j) {
                double s2 = 0.0;
                for (int k = 0; k < DIM; ++k) s2 += G[i * M + k] * a[j * M + k] + a[k * M + i] * G[k * M + j];
                s2 += G[i * M + DIM] * a[j * M + DIM];
                o[i * M + j] += h * G[i * M + j] + hh * s2;
            }
            double s3 = 0.0;
            for (int k = 0; k < DIM; ++k) s3 += a[k * M + i] * G[k * M + DIM];
            o[i * M + DIM] += h * G[i * M + DIM] + hh * s3;
        }
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

template <int DIM, int TESS>
static cudaError_t launch_grad_ref_t(const GradArgs &a, cudaStream_t s)
{
    constexpr int NE = DIM * (DIM + 1);
    // gradient sums in shared memory only while all four arrays stay within 48 KB
    const bool sacc = (size_t)4 * a.t.nC * NE * sizeof(double) <= 48 * 1024;
    size_t smem = (size_t)(sacc ? 4 : 2) * a.t.nC * NE * sizeof(double);
    auto kern = sacc ? k_grad_ref<DIM, TESS, true> : k_grad_ref<DIM, TESS, false>;
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
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int total = a.N * a.t.nC;
    k_frechet_adjoint<DIM><<<(total + 63) / 64, 64, 0, s>>>(a.A, a.gT, a.gA, total, a.dt);
    return cudaGetLastError();
}

template <int DIM, int TESS>
static cudaError_t launch_grad_ref_f32_t(const GradArgs &a, cudaStream_t s)
{
    constexpr int NE = DIM * (DIM + 1);
    const size_t tables = (size_t)2 * a.t.nC * NE * sizeof(float), sums = (size_t)2 * a.t.nC * NE * sizeof(double);
    const bool sacc = tables + sums <= 48 * 1024;
    const size_t smem = tables + (sacc ? sums : 0);
    auto kern = sacc ? k_grad_ref_f32<DIM, TESS, true> : k_grad_ref_f32<DIM, TESS, false>;
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
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int total = a.N * a.t.nC;
    k_frechet_adjoint<DIM><<<(total + 63) / 64, 64, 0, s>>>(a.A, a.gT, a.gA, total, a.dt);
    k_substep_map_adjoint<DIM><<<(total + 127) / 128, 128, 0, s>>>(a.A, a.gS, a.gA, total, a.h_sub);
    return cudaGetLastError();
}

cudaError_t launch_grad_ref_f32(const GradArgs &a, cudaStream_t s)
{
    const int dim = a.t.dim, tess = a.t.tess;
    if (dim == 1) return launch_grad_ref_f32_t<1, 2>(a, s);
    if (dim == 2) return tess == 1 ? launch_grad_ref_f32_t<2, 1>(a, s) : launch_grad_ref_f32_t<2, 2>(a, s);
    return tess == 1 ? launch_grad_ref_f32_t<3, 1>(a, s) : launch_grad_ref_f32_t<3, 2>(a, s);
}

cudaError_t launch_grad_ref(const GradArgs &a, cudaStream_t s)
{
    const int dim = a.t.dim, tess = a.t.tess;
    if (dim == 1) return launch_grad_ref_t<1, 2>(a, s);
    if (dim == 2) return tess == 1 ? launch_grad_ref_t<2, 1>(a, s) : launch_grad_ref_t<2, 2>(a, s);
    return tess == 1 ? launch_grad_ref_t<3, 1>(a, s) : launch_grad_ref_t<3, 2>(a, s);
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
