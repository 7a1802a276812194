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

// Closed-form step with the table of cell c; kept (returns true) if the end
// point is still in cell c.
// cq receives the cell of the end point (equal to c when kept).
template <int DIM, int TESS>
__device__ __forceinline__ bool try_fast(const Tess &t, PState<DIM, double> &s, const double *T, int tab, int c,
                                         int &cq)
{
    double q[DIM];
    exact_affine<DIM>(q, T + c * DIM * (DIM + 1), s.p);
    cq = exact_cell<DIM, TESS>(t, q);
    if (cq != c) return false;
#pragma unroll
    for (int i = 0; i < DIM; ++i) s.p[i] = q[i];
    return true;
}
template <int DIM, int TESS>
__device__ __forceinline__ bool try_fast(const Tess &t, PState<DIM, float> &s, const float *T, int tab, int c,
                                         int &cq)
{
    constexpr int NH = DIM + 1;
    const float *Th = T + c * DIM * NH, *Tl = Th + tab;
    PState<DIM, float> q;
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        // d = (T - I)[r] . [p; 1], hi and lo parts of the table, hi + lo of p
        float d = Th[r * NH + DIM] + Tl[r * NH + DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            d = fmaf(Th[r * NH + k], s.hi[k], d);
            d = fmaf(Tl[r * NH + k], s.hi[k], d);
            d = fmaf(Th[r * NH + k], s.lo[k], d);
        }
        q.hi[r] = s.hi[r];
        q.lo[r] = s.lo[r];
        acc_add(q.hi[r], q.lo[r], d);
    }
    cq = fast_cell<DIM, TESS>(t, q.hi);
    if (cq != c) return false;
    s = q;
    return true;
}

template <int DIM>
__device__ __forceinline__ void substep(PState<DIM, double> &s, const double *A, double h)
{
    exact_midpoint<DIM>(s.p, A, h);
}
template <int DIM>
__device__ __forceinline__ void substep(PState<DIM, float> &s, const float *A, float h)
{
    float v[DIM], pm[DIM];
    fast_affine<DIM>(v, A, s.hi);
    const float hh = 0.5f * h;
#pragma unroll
    for (int i = 0; i < DIM; ++i) pm[i] = fmaf(hh, v[i], s.hi[i]);
    fast_affine<DIM>(v, A, pm);
#pragma unroll
    for (int i = 0; i < DIM; ++i) acc_add(s.hi[i], s.lo[i], h * v[i]);
}

// ------------------------------------------------------------ integration

// One warp integrates the points [ws, we).  Every lane owns one point and
// advances it by one unit per iteration -- a closed-form Trel step or one
// midpoint sub-step, which cost about the same -- and claims the next
// unprocessed point of the range as soon as its own is finished.  A point
// that falls back to nStepsODE sub-steps therefore keeps one lane busy, not
// the whole warp.  Results do not depend on the schedule: each point follows
// exactly the reference's sequence of operations.
//   Src::load(idx, st)     sets the start state of point idx
//   Snk::put(idx, st)      receives the end state (PState; get() converts)
//   perm (optional, shared memory): the k-th point of the range is
//   ws_base + perm[k - ws_base] (a cell-sorted order inside the tile).
//   claim (optional, shared memory, zero on entry): all warps of the CTA
//   share one queue over [ws, we) -- a warp whose lanes finish claims the next
//   points of the whole tile, so no warp idles at the end-of-tile barrier
//   while another still works through a fixed slice.
// The reference recomputes the start cell of every time step; after a kept
// closed-form step that cell was just computed for the same point, so it is
// reused (identical value, one lookup per step saved).
template <int DIM, int TESS, typename Real, int SCHEME, class Src, class Snk>
__device__ __forceinline__ void integrate_range(const Tess &t, int nT, int nODE, const Real *sA, const Real *sT,
                                                int64_t ws, int64_t we, Real h, const Src &src, Snk &snk,
                                                unsigned long long &c_fast, unsigned long long &c_fb,
                                                unsigned long long &c_sub, unsigned long long &c_pts,
                                                const int *perm = nullptr, int64_t perm_base = 0,
                                                unsigned long long *claim = nullptr)
{
    constexpr int NE = DIM * (DIM + 1);
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
    int steps_left = 0, sub_left = 0, known_cell = -1;
    if (active) {
        src.load(idx, st);
        steps_left = nT;
        sub_left = (SCHEME == SCHEME_SIMPLE) ? nT * nODE : 0;
    }
    while (__any_sync(FULL, active)) {
        bool fin = false;
        if (active) {
            if (SCHEME == SCHEME_REF && sub_left == 0) {
                const int c = known_cell >= 0 ? known_cell : cell_of<DIM, TESS>(t, st);
                int cq;
                if (try_fast<DIM, TESS>(t, st, sT, tab, c, cq)) {
                    --steps_left;
                    ++c_fast;
                    known_cell = cq;
                } else {
                    sub_left = nODE;
                    ++c_fb;
                    known_cell = -1;
                }
            } else {
                const int c = cell_of<DIM, TESS>(t, st);
                substep<DIM>(st, sA + c * NE, h);
                --sub_left;
                ++c_sub;
                if (sub_left == 0) --steps_left;
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
                    steps_left = nT;
                    sub_left = (SCHEME == SCHEME_SIMPLE) ? nT * nODE : 0;
                    known_cell = -1;
                }
            }
            next += __popc(done);
        }
    }
}

}  // namespace cpab
