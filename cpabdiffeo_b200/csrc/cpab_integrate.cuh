// cpab_integrate.cuh -- the integration arithmetic (exact double / fast
// float overloads) and the lane-scheduled warp loop shared by k_integrate
// (calc_T) and the fused registration likelihood.
#pragma once

#include "cpab_device.cuh"

namespace cpab {

// ------------------------------------------------------------ arithmetic
//
// Two per-point states:
//  * double (bit-exact family): one double per coordinate, the reference's
//    arithmetic (cpab_cell.cuh).
//  * float (FP32 mode): a compensated pair hi + lo per coordinate (TwoSum,
//    Knuth), so the many small increments of the integration are not lost to
//    float rounding; velocities and cell lookups use hi.  The closed-form
//    step table holds T - I split into a float pair (hi, lo), so rounding T to
//    float does not bias every step; the velocity table A is plain float.
// Shared-memory tables per cell:
//  double: A[ne], T[ne];   float: A[ne], (T-I)_hi[ne], (T-I)_lo[ne].

template <int DIM, typename Real>
struct PState;

template <int DIM>
struct PState<DIM, double> {
    double p[DIM];
    __device__ __forceinline__ void set(const double *x)
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) p[i] = x[i];
    }
    __device__ __forceinline__ void get(double *x) const
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) x[i] = p[i];
    }
    __device__ __forceinline__ const double *lookup() const { return p; }
};

template <int DIM>
struct PState<DIM, float> {
    float hi[DIM], lo[DIM];
    __device__ __forceinline__ void set(const float *x)
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) { hi[i] = x[i]; lo[i] = 0.0f; }
    }
    __device__ __forceinline__ void set(const double *x)
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) { hi[i] = (float)x[i]; lo[i] = (float)(x[i] - (double)hi[i]); }
    }
    __device__ __forceinline__ void get(float *x) const
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) x[i] = hi[i] + lo[i];
    }
    __device__ __forceinline__ void get(double *x) const
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) x[i] = (double)hi[i] + (double)lo[i];
    }
    __device__ __forceinline__ const float *lookup() const { return hi; }
};

// s + e == a + b exactly (Knuth's TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e)
{
    s = a + b;
    float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// (hi, lo) += d, renormalised.
__device__ __forceinline__ void acc_add(float &hi, float &lo, float d)
{
    float s, e;
    two_sum(hi, d, s, e);
    e += lo;
    hi = s + e;
    lo = e - (hi - s);
}

template <typename Real>
struct TableLayout {
    // floats per cell of the closed-form table (double: T; float: (T-I) hi and lo)
    static constexpr int kTParts = sizeof(Real) == 8 ? 1 : 2;
};

// Stage one instance's tables in shared memory.
template <int DIM, typename Real>
__device__ __forceinline__ void stage_tables(const double *gA, const double *gT, int nC, bool with_T, Real *sA,
                                             Real *sT)
{
    constexpr int NE = DIM * (DIM + 1);
    const int tab = nC * NE;
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        sA[i] = (Real)gA[i];
        if (with_T) {
            if (sizeof(Real) == 8) {
                sT[i] = (Real)gT[i];
            } else {
                const int e = i % NE, r = e / (DIM + 1), c = e % (DIM + 1);
                const double d = gT[i] - (r == c ? 1.0 : 0.0);
                const float hi = (float)d;
                sT[i] = hi;
                sT[tab + i] = (float)(d - (double)hi);
            }
        }
    }
}

template <int DIM, int TESS>
__device__ __forceinline__ int cell_of(const Tess &t, const PState<DIM, double> &s)
{
    return exact_cell<DIM, TESS>(t, s.p);
}
template <int DIM, int TESS>
__device__ __forceinline__ int cell_of(const Tess &t, const PState<DIM, float> &s)
{
    return fast_cell<DIM, TESS>(t, s.hi);
}

// One unit of work on a point in cell c: the candidate end point q of a
// closed-form step (fast: q = T_c [p; 1]) or of one explicit-midpoint
// sub-step with A_c.  The caller looks up the cell of q; a closed-form step
// is kept when that is still c (calc_2Dto2D.cu:380-400), a sub-step always
// is, and its end cell is the cell of the next sub-step's start point.
//   double: the reference's arithmetic (exact_affine / exact_midpoint).
//   float:  both kinds share the first matrix-vector product (T - I)_hi [p; 1]
//           resp. A [p; 1] and the compensated update, so a warp whose lanes
//           mix closed-form steps and sub-steps diverges only in between.
template <int DIM>
__device__ __forceinline__ void advance(bool fast, const PState<DIM, double> &s, const double *A, const double *T,
                                        const double *, double h, PState<DIM, double> &q)
{
    if (fast) {
        exact_affine<DIM>(q.p, T, s.p);
    } else {
        q = s;
        exact_midpoint<DIM>(q.p, A, h);
    }
}
template <int DIM>
__device__ __forceinline__ void advance(bool fast, const PState<DIM, float> &s, const float *A, const float *Th,
                                        const float *Tl, float h, PState<DIM, float> &q)
{
    constexpr int NH = DIM + 1;
    float y[DIM], d[DIM];
    fast_affine<DIM>(y, fast ? Th : A, s.hi);
    if (fast) {
        // d = (T - I)[p; 1] with the lo table and the lo part of p: small terms first
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
            float e = Tl[r * NH + DIM];
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                e = fmaf(Tl[r * NH + k], s.hi[k], e);
                e = fmaf(Th[r * NH + k], s.lo[k], e);
            }
            d[r] = y[r] + e;
        }
    } else {
        float pm[DIM];
        const float hh = 0.5f * h;
#pragma unroll
        for (int i = 0; i < DIM; ++i) pm[i] = fmaf(hh, y[i], s.hi[i]);
        fast_affine<DIM>(y, A, pm);
#pragma unroll
        for (int i = 0; i < DIM; ++i) d[i] = h * y[i];
    }
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        q.hi[r] = s.hi[r];
        q.lo[r] = s.lo[r];
        acc_add(q.hi[r], q.lo[r], d[r]);
    }
}

// ------------------------------------------------------------ integration

// One warp integrates the points [ws, we).  Every lane owns one point and
// advances it by one unit per iteration -- a closed-form Trel step or one
// midpoint sub-step, which cost about the same and share most of their
// instructions (advance) -- and claims the next unprocessed point of the
// range as soon as its own is finished.  A point that falls back to
// nStepsODE sub-steps therefore keeps one lane busy, not the whole warp.
// Results do not depend on the schedule: each point follows exactly the
// reference's sequence of operations.
//   Src::load(idx, st)     sets the start state of point idx
//   Snk::put(idx, st)      receives the end state (PState; get() converts)
//   perm (optional, shared memory): the k-th point of the range is
//   ws_base + perm[k - ws_base] (a cell-sorted order inside the tile).
//   claim (optional, shared memory, zero on entry): all warps of the CTA
//   share one queue over [ws, we) -- a warp whose lanes finish claims the next
//   points of the whole tile, so no warp idles at the end-of-tile barrier
//   while another still works through a fixed slice.
// Every iteration ends with one cell lookup, of the candidate end point: for
// a closed-form step it is the reference's keep test, for a sub-step it is
// the cell the next sub-step (or the next time step) starts in, which the
// reference would look up from the same point.  So each lane always knows
// the cell of its current point.
template <int DIM, int TESS, typename Real, int SCHEME, class Src, class Snk>
__device__ __forceinline__ void integrate_range(const Tess &t, int nT, int nODE, const Real *sA, const Real *sT,
                                                int64_t ws, int64_t we, Real h, const Src &src, Snk &snk,
                                                unsigned long long &c_fast, unsigned long long &c_fb,
                                                unsigned long long &c_sub, unsigned long long &c_pts,
                                                const int *perm = nullptr, int64_t perm_base = 0,
                                                unsigned long long *claim = nullptr)
{
    constexpr int NE = DIM * (DIM + 1);
    constexpr bool kTwoPart = TableLayout<Real>::kTParts == 2;
    const int tab = t.nC * NE;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int64_t next = ws + 32;
    int64_t k;
    if (claim) {
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(claim, 32ull);
        k = ws + (int64_t)__shfl_sync(FULL, b, 0) + lane;
    } else {
        k = ws + lane;
    }
    bool active = k < we;
    int64_t idx = (active && perm) ? perm_base + perm[k - perm_base] : k;
    PState<DIM, Real> st;
    int steps_left = 0, sub_left = 0, c = 0;
    if (active) {
        src.load(idx, st);
        c = cell_of<DIM, TESS>(t, st);
        steps_left = nT;
        sub_left = (SCHEME == SCHEME_SIMPLE) ? nT * nODE : 0;
    }
    while (__any_sync(FULL, active)) {
        bool fin = false;
        if (active) {
            const bool fast = (SCHEME == SCHEME_REF) && sub_left == 0;
            PState<DIM, Real> q;
            advance<DIM>(fast, st, sA + c * NE, sT + c * NE, kTwoPart ? sT + tab + c * NE : nullptr, h, q);
            const int cq = cell_of<DIM, TESS>(t, q);
            if (fast && cq != c) {
                // the end point left the cell: redo the step with nStepsODE sub-steps from p
                sub_left = nODE;
                ++c_fb;
            } else {
                st = q;
                c = cq;
                if (fast) {
                    --steps_left;
                    ++c_fast;
                } else {
                    --sub_left;
                    ++c_sub;
                    if (SCHEME == SCHEME_REF && sub_left == 0) --steps_left;
                }
            }
            fin = (SCHEME == SCHEME_SIMPLE) ? (sub_left == 0) : (steps_left == 0);
            if (fin) {
                snk.put(idx, st);
                ++c_pts;
            }
        }
        unsigned done = __ballot_sync(FULL, fin);
        if (done) {
            int64_t base;
            if (claim) {
                unsigned long long b = 0;
                if (lane == 0) b = atomicAdd(claim, (unsigned long long)__popc(done));
                base = ws + (int64_t)__shfl_sync(FULL, b, 0);
            } else {
                base = next;
            }
            if (fin) {
                k = base + __popc(done & lt);
                active = k < we;
                if (active) {
                    idx = perm ? perm_base + perm[k - perm_base] : k;
                    src.load(idx, st);
                    c = cell_of<DIM, TESS>(t, st);
                    steps_left = nT;
                    sub_left = (SCHEME == SCHEME_SIMPLE) ? nT * nODE : 0;
                }
            }
            next += __popc(done);
        }
    }
}

}  // namespace cpab
