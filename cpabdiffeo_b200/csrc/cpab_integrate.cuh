// cpab_integrate.cuh -- the integration arithmetic (exact double / fast
// float overloads) and the lane-scheduled warp loop shared by k_integrate
// (calc_T) and the fused registration likelihood.
#pragma once

#include <math_constants.h>

#include "cpab_device.cuh"

namespace cpab {

// ------------------------------------------------------------ arithmetic
//
// Two per-point states:
//  * double (bit-exact family): one double per coordinate, the reference's
//    arithmetic (cpab_cell.cuh).
//  * float (FP32 mode): an unnormalised compensated pair hi + lo per
//    coordinate plus x = fl(hi + lo), the float nearest the point, which the
//    velocity, the closed-form step and the cell lookup read.  Each update
//    adds its increment d to hi and the rounding error of that addition
//    (Fast2Sum; |d| is a small step, and where |hi| < |d| the error term is
//    below ulp(d)) to lo, so the many small increments of the integration are
//    not lost to float rounding.  Both step kinds are increments from a
//    small matrix: the closed-form step adds (T - I)[x; 1]; an explicit
//    midpoint sub-step of length h with the cell's velocity v(x) = A[x; 1]
//    (both evaluations in the cell of x, calc_2Dto2D.cu:177-196) is, inside
//    one cell, the affine map x + h v(x + h/2 v(x)) = x + (S - I)[x; 1] with
//        S - I = [h L + h^2/2 L^2 | h b + h^2/2 L b]      (A = [L | b]),
//    evaluated in double when the tables are staged.  Table roundings are
//    relative to the small increments, not to the position, so they do not
//    bias every step.
// Shared-memory tables per cell (ne = DIM * (DIM + 1)):
//  double: A[ne], T[ne], row-major as in global memory;
//  float:  (S - I)[ne] and (T - I)[ne], column-major (the DIM columns of the
//          linear part, then the offset) so that a cell's matrix is read with
//          8-byte (1D/2D) or 16-byte (3D) loads.

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
    float hi[DIM], lo[DIM], x[DIM];
    __device__ __forceinline__ void set(const float *v)
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) { hi[i] = v[i]; lo[i] = 0.0f; x[i] = v[i]; }
    }
    __device__ __forceinline__ void set(const double *v)
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) {
            hi[i] = (float)v[i];
            lo[i] = (float)(v[i] - (double)hi[i]);
            x[i] = hi[i] + lo[i];
        }
    }
    __device__ __forceinline__ void get(float *v) const
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) v[i] = x[i];
    }
    __device__ __forceinline__ void get(double *v) const
    {
#pragma unroll
        for (int i = 0; i < DIM; ++i) v[i] = (double)hi[i] + (double)lo[i];
    }
    __device__ __forceinline__ const float *lookup() const { return x; }
    // hi + lo += d
    __device__ __forceinline__ void add(int i, float d)
    {
        const float s = hi[i] + d;
        lo[i] += d - (s - hi[i]);
        hi[i] = s;
        x[i] = s + lo[i];
    }
};

template <typename Real>
struct TableLayout {
    // tables of the closed-form step per cell (double: T; float: T - I)
    static constexpr int kTParts = 1;
};

// Stage one instance's tables in shared memory (layout above); h is the
// sub-step length dt / nStepsODE (float tables only), passed from the
// kernel's parameters so that no register holds it during integration.
// EXACT scheme (2D/3D): the sub-step map is the exact flow S = expm(h A)
// instead of the midpoint map, staged by stage_exact_substeps below.
template <int DIM, typename Real>
__device__ void stage_exact_substeps(const double *gA, const double *gT, int nC, double h, Real *sS, Real *sT);

template <int DIM, typename Real>
__device__ __forceinline__ void stage_tables(const double *gA, const double *gT, int nC, bool with_T, double h,
                                             Real *sA, Real *sT, bool exact_sub = false)
{
    constexpr int NE = DIM * (DIM + 1);
    const int tab = nC * NE;
    if (exact_sub) {
        stage_exact_substeps<DIM, Real>(gA, gT, nC, h, sA, sT);
        return;
    }
    // not unrolled: the staging loop's loads in flight would otherwise set
    // the register count of the integration loop that follows
#pragma unroll 1
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        if (sizeof(Real) == 8) {
            sA[i] = (Real)gA[i];
            if (with_T) sT[i] = (Real)gT[i];
        } else {
            const int c = i / NE, e = i - c * NE, r = e / (DIM + 1), col = e - r * (DIM + 1);
            const int cm = col * DIM + r;
            // (S - I)[r][col] = h (A[r][col] + h/2 sum_k L[r][k] A[k][col])
            const double *a = gA + (size_t)c * NE;
            double l2 = 0.0;
#pragma unroll 1
            for (int k = 0; k < DIM; ++k) l2 += a[r * (DIM + 1) + k] * a[k * (DIM + 1) + col];
            sA[c * NE + cm] = (float)(h * (a[r * (DIM + 1) + col] + 0.5 * h * l2));
            if (with_T) sT[c * NE + cm] = (float)(gT[i] - (r == col ? 1.0 : 0.0));
        }
    }
}

// A cell's column-major float matrix into registers (8-byte loads in 1D/2D,
// 16-byte loads in 3D; the tables' offsets keep those aligned).
template <int DIM>
__device__ __forceinline__ void load_cell(const float *p, float *m)
{
    constexpr int NE = DIM * (DIM + 1);
    if (DIM == 3) {
#pragma unroll
        for (int i = 0; i < NE / 4; ++i) {
            const float4 v = reinterpret_cast<const float4 *>(p)[i];
            m[4 * i] = v.x;
            m[4 * i + 1] = v.y;
            m[4 * i + 2] = v.z;
            m[4 * i + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < NE / 2; ++i) {
            const float2 v = reinterpret_cast<const float2 *>(p)[i];
            m[2 * i] = v.x;
            m[2 * i + 1] = v.y;
        }
    }
}

// y = M [x; 1] for a column-major cell matrix held in registers
template <int DIM>
__device__ __forceinline__ void cm_affine(float *y, const float *m, const float *x)
{
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        float acc = m[DIM * DIM + r];
#pragma unroll
        for (int k = 0; k < DIM; ++k) acc = fmaf(m[k * DIM + r], x[k], acc);
        y[r] = acc;
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
    return fast_cell<DIM, TESS>(t, s.x);
}

// One unit of work on a point in cell c: the candidate end point q of a
// closed-form step (fast: q = T_c [p; 1]) or of one explicit-midpoint
// sub-step with A_c.  The caller looks up the cell of q; a closed-form step
// is kept when that is still c (calc_2Dto2D.cu:380-400), a sub-step always
// is, and its end cell is the cell of the next sub-step's start point.
//   double: the reference's arithmetic (exact_affine / exact_midpoint).
//   float:  one matrix-vector product with the cell's (T - I) or (S - I)
//           and the compensated update -- the same instructions for both
//           kinds, so lanes that mix closed-form steps and sub-steps do not
//           diverge.
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
// Paired FP32 arithmetic (sm_100's FFMA2 / FADD2: two lanes of float math per
// instruction, each rounded as its scalar twin) for the (x, y) coordinates:
// the column-major cell matrix gives column k as the pair (M[0][k], M[1][k]).
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// hi + lo += d for coordinates 0 and 1 at once (PState::add, twice)
template <int DIM>
__device__ __forceinline__ void add_pair(PState<DIM, float> &q, float2 d)
{
    const float2 hi = make_float2(q.hi[0], q.hi[1]), lo = make_float2(q.lo[0], q.lo[1]);
    const float2 sm = __fadd2_rn(hi, d);
    const float2 l2 = __fadd2_rn(lo, __fadd2_rn(d, neg2(__fadd2_rn(sm, neg2(hi)))));
    const float2 x = __fadd2_rn(sm, l2);
    q.hi[0] = sm.x; q.hi[1] = sm.y;
    q.lo[0] = l2.x; q.lo[1] = l2.y;
    q.x[0] = x.x; q.x[1] = x.y;
}

template <int DIM>
__device__ __forceinline__ void advance(bool fast, const PState<DIM, float> &s, const float *A, const float *T,
                                        const float *, float, PState<DIM, float> &q)
{
    constexpr int NE = DIM * (DIM + 1);
    float m[NE], d[DIM];
    // d = (T - I)[x; 1] for a closed-form step, (S - I)[x; 1] for a sub-step
    load_cell<DIM>(fast ? T : A, m);
    q = s;
    if constexpr (DIM == 1) {
        cm_affine<DIM>(d, m, s.x);
        q.add(0, d[0]);
    } else {
        // rows 0 and 1 as one pair: the same fmaf sequence as cm_affine per row
        float2 d01 = make_float2(m[DIM * DIM], m[DIM * DIM + 1]);
#pragma unroll
        for (int k = 0; k < DIM; ++k)
            d01 = __ffma2_rn(make_float2(m[k * DIM], m[k * DIM + 1]), make_float2(s.x[k], s.x[k]), d01);
        add_pair<DIM>(q, d01);
        if constexpr (DIM == 3) {
            float d2 = m[DIM * DIM + 2];
#pragma unroll
            for (int k = 0; k < DIM; ++k) d2 = fmaf(m[k * DIM + 2], s.x[k], d2);
            q.add(2, d2);
        }
    }
}

// ------------------------------------------------------------ exact scheme (2D/3D)
//
// Sub-step map of the exact flow: column j of S - I is
// sum_{k>=1} h^k/k! L^{k-1} A[:, j]  (A = [L | b], homogeneous bottom row 0),
// summed per column until the terms fall below the sum's rounding.
// double tables: S row-major (the layout exact_affine-style code reads);
// float tables: S - I column-major (the layout of the float sub-step table).
template <int DIM, typename Real>
__device__ void stage_exact_substeps(const double *gA, const double *gT, int nC, double h, Real *sS, Real *sT)
{
    constexpr int NE = DIM * (DIM + 1);
#pragma unroll 1
    for (int c = threadIdx.x; c < nC; c += blockDim.x) {
        const double *a = gA + (size_t)c * NE;
        double L[DIM * DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int k = 0; k < DIM; ++k) L[r * DIM + k] = a[r * (DIM + 1) + k];
#pragma unroll 1
        for (int col = 0; col <= DIM; ++col) {
            double w[DIM], acc[DIM];
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
                w[r] = h * a[r * (DIM + 1) + col];
                acc[r] = w[r];
            }
#pragma unroll 1
            for (int k = 2; k <= 40; ++k) {
                double nw[DIM], big = 0.0, am = 0.0;
#pragma unroll
                for (int r = 0; r < DIM; ++r) {
                    double v = 0.0;
#pragma unroll
                    for (int m = 0; m < DIM; ++m) v = fma(L[r * DIM + m], w[m], v);
                    nw[r] = v * (h / k);
                }
#pragma unroll
                for (int r = 0; r < DIM; ++r) {
                    w[r] = nw[r];
                    acc[r] += w[r];
                    big = fmax(big, fabs(w[r]));
                    am = fmax(am, fabs(acc[r]));
                }
                if (!(big > 1e-18 * am)) break;
            }
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
                if (sizeof(Real) == 8)
                    sS[c * NE + r * (DIM + 1) + col] = (Real)(acc[r] + (r == col ? 1.0 : 0.0));
                else
                    sS[c * NE + col * DIM + r] = (Real)acc[r];
            }
        }
    }
    const int tab = nC * NE;
#pragma unroll 1
    for (int i = threadIdx.x; i < tab; i += blockDim.x) {
        if (sizeof(Real) == 8) {
            sT[i] = (Real)gT[i];
        } else {
            const int c = i / NE, e = i - c * NE, r = e / (DIM + 1), col = e - r * (DIM + 1);
            sT[c * NE + col * DIM + r] = (Real)(gT[i] - (r == col ? 1.0 : 0.0));
        }
    }
}

// What a lane needs to resolve an exit: the instance's signed A (global,
// row-major [nC, DIM*(DIM+1)]), the facet tables, the sub-step length and
// the lane's counters.
// Parked exits a warp resolves together, and the votes the oldest may wait
// (integrate_range).
#ifndef CPAB_EXACT_CROSS_BATCH
#define CPAB_EXACT_CROSS_BATCH 16
#endif
#ifndef CPAB_EXACT_CROSS_WAIT
#define CPAB_EXACT_CROSS_WAIT 96
#endif

struct ExactCross {
    const double *A;
    const double *F;
    const int *nbr;
    int nF;
    double h;
    int cap;
    unsigned long long crossings, unresolved;
};

template <int DIM, int TESS>
__device__ __forceinline__ int lookup_d(const Tess &t, const double *p, double)
{
    return exact_cell<DIM, TESS>(t, p);
}
template <int DIM, int TESS>
__device__ __forceinline__ int lookup_d(const Tess &t, const double *p, float)
{
    float x[DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i) x[i] = (float)p[i];
    return fast_cell<DIM, TESS>(t, x);
}

// The flow inside a cell over a time t <= h (one sub-step) as a Taylor
// polynomial: x(t) = p + sum_{k>=1} w_k, w_k = t^k/k! u_k, u_1 = L p + b,
// u_k = L u_{k-1} (A = [L | b], read through the read-only cache at each use:
// held in registers it raised the kernel's spills, 37.3 against 36.1 ms).  The
// series stops at the first degree K whose omitted terms are provably below
// FP64 rounding of the first: with r = t |L| / (K+1) < 1 (|L| the max row
// sum), |w_{K+j}| <= |w_K| r^j, so the rest sums to at most |w_K| r/(1-r).
// At sub-step lengths (t |L| ~ 1e-3) that is K = 6 or 7; kExactDeg caps it,
// and a flow the cap does not resolve (t |L| above ~0.1) is reported so that
// exact_substep_cross keeps the reference scheme's sub-step end.
constexpr int kExactDeg = 10;
constexpr double kTaylorTol = 1e-17;
// 1/k for the Taylor recurrences (a product instead of an FP64 division per term)
static __constant__ double kInvInt[kExactDeg + 2] = {0.0,       1.0,       1.0 / 2,  1.0 / 3,
                                                     1.0 / 4,   1.0 / 5,   1.0 / 6,  1.0 / 7,
                                                     1.0 / 8,   1.0 / 9,   1.0 / 10, 1.0 / 11};

template <int DIM>
__device__ __forceinline__ double affine_norm(const double *__restrict__ A)
{
    double lnorm = 0.0;
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        double rs = 0.0;
#pragma unroll
        for (int m = 0; m < DIM; ++m) rs += fabs(__ldg(A + r * (DIM + 1) + m));
        lnorm = fmax(lnorm, rs);
    }
    return lnorm;
}

template <int DIM>
__device__ __forceinline__ void affine_lin(const double *__restrict__ A, const double *u, double *out)
{
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        double v = 0.0;
#pragma unroll
        for (int m = 0; m < DIM; ++m) v = fma(__ldg(A + r * (DIM + 1) + m), u[m], v);
        out[r] = v;
    }
}

template <int DIM>
__device__ __forceinline__ void velocity(const double *__restrict__ A, const double *p, double *v)
{
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        double s = __ldg(A + r * (DIM + 1) + DIM);
#pragma unroll
        for (int m = 0; m < DIM; ++m) s = fma(__ldg(A + r * (DIM + 1) + m), p[m], s);
        v[r] = s;
    }
}

// out = expm(t A)[p; 1] (out may alias p); false when kExactDeg terms do
// not bring the omitted rest below FP64 rounding of the first term
template <int DIM>
__device__ __forceinline__ bool flow_taylor(const double *__restrict__ A, const double *p, double t, double *out)
{
    const double *Ar = A;  // global, read through __ldg
    const double lnorm = affine_norm<DIM>(A);
    double u[DIM], x[DIM];
    velocity<DIM>(Ar, p, u);
    double coef = t, first = 0.0;
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        x[r] = fma(coef, u[r], p[r]);
        first = fmax(first, fabs(coef * u[r]));
    }
    const double tl = fabs(t) * lnorm;
    bool ok = false;
#pragma unroll 1
    for (int k = 2; k <= kExactDeg; ++k) {
        double nu[DIM];
        affine_lin<DIM>(Ar, u, nu);
        coef *= t * kInvInt[k];
        double wk = 0.0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
            u[r] = nu[r];
            x[r] = fma(coef, u[r], x[r]);
            wk = fmax(wk, fabs(coef * u[r]));
        }
        const double rr = tl * kInvInt[k + 1];
        if (rr < 0.5 && wk * rr <= kTaylorTol * (1.0 - rr) * first) {
            ok = true;
            break;
        }
    }
#pragma unroll
    for (int r = 0; r < DIM; ++r) out[r] = x[r];
    return ok || first == 0.0;
}

// First root in [0, s] of g(t) = F . x(t) + F[DIM] along the flow of A from
// p, given g(0) = g0 < 0 < g(s): the Taylor coefficients of g,
// c_k = F . u_k / k!, up to the degree whose omitted rest is below FP64
// rounding of g over [0, s] (the bound of flow_taylor times |F|_1), and a
// safeguarded Newton iteration on that polynomial.  Returns NaN when
// kExactDeg terms do not resolve g to that rounding.
template <int DIM>
__device__ __forceinline__ double facet_hit_time(const double *__restrict__ A, const double *__restrict__ F,
                                                 const double *p, double s, double g0)
{
    const double *Ar = A;  // global, read through __ldg
    const double lnorm = affine_norm<DIM>(A);
    double c[kExactDeg + 1];
    c[0] = g0;
    double u[DIM], Fn[DIM], f1 = 0.0;
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        Fn[r] = __ldg(F + r);
        f1 += fabs(Fn[r]);
    }
    velocity<DIM>(Ar, p, u);
    const double sl = s * lnorm;
    double inv_fact = 1.0, sk = 1.0, scale = 0.0;
    int K = 0;
#pragma unroll 1
    for (int k = 1; k <= kExactDeg; ++k) {
        if (k > 1) {
            double nu[DIM];
            affine_lin<DIM>(Ar, u, nu);
#pragma unroll
            for (int r = 0; r < DIM; ++r) u[r] = nu[r];
        }
        inv_fact *= kInvInt[k];
        sk *= s;
        double d = 0.0, un = 0.0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
            d = fma(Fn[r], u[r], d);
            un = fmax(un, fabs(u[r]));
        }
        c[k] = d * inv_fact;
        if (k == 1) {
            scale = fabs(g0) + fabs(c[1]) * s;
        } else {
            const double rr = sl * kInvInt[k + 1];
            if (rr < 0.5 && f1 * un * inv_fact * sk * rr <= kTaylorTol * (1.0 - rr) * scale) {
                K = k;
                break;
            }
        }
    }
    if (K == 0) return CUDART_NAN;
    auto P = [&](double t, double &dP) {
        double v = c[K], dv = 0.0;
#pragma unroll 1
        for (int k = K - 1; k >= 0; --k) {
            dv = fma(dv, t, v);
            v = fma(v, t, c[k]);
        }
        dP = dv;
        return v;
    };
    double lo = 0.0, hi = s, dP;
    const double ps = P(s, dP);
    if (!(ps > 0)) return s;
    double t = s * (-g0) / (ps - g0);
    if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
#pragma unroll 1
    for (int it = 0; it < 60; ++it) {
        const double g = P(t, dP);
        if (g > 0) hi = t; else lo = t;
        if (g == 0) return t;
        double tn = t - g / dP;
        if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
        // converged within about two ulps (4.5e-16 relative is at least two
        // ulps in every binade: a tolerance under one ulp never ends an
        // iteration that alternates between neighbouring doubles)
        if (fabs(tn - t) <= 4.5e-16 * fabs(t) || hi - lo <= 4.5e-16 * hi) return tn;
        t = tn;
    }
    return 0.5 * (lo + hi);
}

// A sub-step of length h from st in cell c ended at q outside c: the exact
// flow from st, exit times through interior facets, the neighbour across the
// exited facet, the rest of the sub-step there (and so on).  q becomes the
// point at the sub-step's end; returns its cell.  FP64 throughout (the
// hitting times); q keeps the state's precision.  When no interior facet
// explains the exit (a point on the domain boundary) or the crossings exceed
// the cap, q is the end point of the flow in the current cell (as in the
// reference scheme, which keeps its sub-step's end wherever it lands).
template <int DIM, int TESS, typename Real>
__device__ __forceinline__ int exact_substep_cross(const Tess &t, ExactCross &ex, int c,
                                                   const PState<DIM, Real> &st, PState<DIM, Real> &q)
{
    constexpr int NH = DIM + 1, NE = DIM * NH;
    double p[DIM], y[DIM];
    st.get(p);
    q.get(y);
    double s = ex.h;
#pragma unroll 1
    for (int crossings = 0;;) {
        // (the caller found q outside c; later ends are looked up here)
        if (crossings > 0 && lookup_d<DIM, TESS>(t, y, Real(0)) == c) {
            q.set(y);
            return c;
        }
        const double *A = ex.A + (size_t)c * NE;
        const double *Fc = ex.F + (size_t)c * ex.nF * NH;
        double tau = s;
        int kbest = -1;
#pragma unroll 1
        for (int k = 0; k < ex.nF; ++k) {
            if (__ldg(ex.nbr + c * ex.nF + k) < 0) continue;
            const double *F = Fc + k * NH;
            double ge = __ldg(F + DIM), g0 = ge;
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
                const double n = __ldg(F + r);
                ge = fma(n, y[r], ge);
                g0 = fma(n, p[r], g0);
            }
            if (!(ge > 0)) continue;
            const double r = (g0 >= 0) ? 0.0 : facet_hit_time<DIM>(A, F, p, s, g0);
            if (kbest < 0 || r < tau) {
                tau = r;
                kbest = k;
            }
        }
        if (kbest < 0 || !(tau == tau) || ++crossings > ex.cap) {
            ++ex.unresolved;
            q.set(y);
            return lookup_d<DIM, TESS>(t, y, Real(0));
        }
        flow_taylor<DIM>(A, p, tau, p);
        s -= tau;
        c = __ldg(ex.nbr + c * ex.nF + kbest);
        ++ex.crossings;
        if (!(s > 0)) {
            q.set(p);
            return c;
        }
        if (!flow_taylor<DIM>(ex.A + (size_t)c * NE, p, s, y)) {
            // the neighbour's flow is too fast for the polynomial over the
            // rest of the sub-step: the reference scheme's sub-step end
            ++ex.unresolved;
            return cell_of<DIM, TESS>(t, q);
        }
    }
}

// EXACT unit: the closed-form step with T (the reference's arithmetic in
// double) or one sub-step of the exact flow with S.
template <int DIM>
__device__ __forceinline__ void advance_exact(bool fast, const PState<DIM, double> &s, const double *S,
                                              const double *T, PState<DIM, double> &q)
{
    if (fast) {
        exact_affine<DIM>(q.p, T, s.p);
    } else {
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
            double v = S[r * (DIM + 1) + DIM];
#pragma unroll
            for (int m = 0; m < DIM; ++m) v = fma(S[r * (DIM + 1) + m], s.p[m], v);
            q.p[r] = v;
        }
    }
}
template <int DIM>
__device__ __forceinline__ void advance_exact(bool fast, const PState<DIM, float> &s, const float *S, const float *T,
                                              PState<DIM, float> &q)
{
    advance<DIM>(fast, s, S, T, nullptr, 0.0f, q);
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
//   start_cells (optional, with perm): cell of point perm_base + i at [i],
//   as computed by the caller's sort pass (same lookup, same point).
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
                                                unsigned long long *claim = nullptr,
                                                const int *start_cells = nullptr, ExactCross *ex = nullptr)
{
    constexpr int NE = DIM * (DIM + 1);
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
        c = start_cells ? start_cells[idx - perm_base] : cell_of<DIM, TESS>(t, st);
        steps_left = nT;
        sub_left = (SCHEME == SCHEME_SIMPLE) ? nT * nODE : 0;
    }
    // FP32: two units per lane between the warp's votes (a lane whose point
    // finishes after the first idles for the second; points finish about once
    // in a hundred units)
    constexpr int kUnits = sizeof(Real) == 4 ? 2 : 1;
    // EXACT: a sub-step that ends outside its cell parks the lane (pend)
    // instead of resolving the exit at once: resolving takes about as long as
    // a hundred units, and done alone it leaves the other 31 lanes idle.  The
    // warp resolves all parked lanes together once kCrossBatch of them wait,
    // every active lane waits, or the oldest has waited kCrossWait votes; a
    // parked lane keeps only the sub-step's start and recomputes its end then
    // (same arithmetic, fewer registers held).  Each point's arithmetic is
    // unchanged.
    constexpr int kCrossBatch = CPAB_EXACT_CROSS_BATCH, kCrossWait = CPAB_EXACT_CROSS_WAIT;
    bool pend = false;
    int pend_votes = 0;
    while (__any_sync(FULL, active)) {
        bool fin = false;
#pragma unroll
        for (int u = 0; u < kUnits; ++u) {
            if (active && !fin && !pend) {
                const bool fast = (SCHEME == SCHEME_REF || SCHEME == SCHEME_EXACT) && sub_left == 0;
                PState<DIM, Real> q;
                if (SCHEME == SCHEME_EXACT)
                    advance_exact<DIM>(fast, st, sA + c * NE, sT + c * NE, q);
                else
                    advance<DIM>(fast, st, sA + c * NE, sT + c * NE, nullptr, h, q);
                int cq = cell_of<DIM, TESS>(t, q);
                if (SCHEME == SCHEME_EXACT && !fast && cq != c) {
                    pend = true;
                    continue;
                }
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
                        if (SCHEME != SCHEME_SIMPLE && sub_left == 0) --steps_left;
                    }
                }
                fin = (SCHEME == SCHEME_SIMPLE) ? (sub_left == 0) : (steps_left == 0);
                if (fin) {
                    snk.put(idx, st);
                    ++c_pts;
                }
            }
        }
        if (SCHEME == SCHEME_EXACT) {
            const unsigned pm = __ballot_sync(FULL, pend);
            if (pm) {
                const unsigned am = __ballot_sync(FULL, active);
                if (__popc(pm) >= kCrossBatch || pm == am || ++pend_votes > kCrossWait) {
                    pend_votes = 0;
                    if (pend) {
                        // the parked sub-step's end, recomputed with the same arithmetic
                        PState<DIM, Real> qp;
                        advance_exact<DIM>(false, st, sA + c * NE, sT + c * NE, qp);
                        c = exact_substep_cross<DIM, TESS, Real>(t, *ex, c, st, qp);
                        st = qp;
                        pend = false;
                        --sub_left;
                        ++c_sub;
                        if (sub_left == 0) --steps_left;
                        fin = steps_left == 0;
                        if (fin) {
                            snk.put(idx, st);
                            ++c_pts;
                        }
                    }
                }
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
                    c = start_cells ? start_cells[idx - perm_base] : cell_of<DIM, TESS>(t, st);
                    steps_left = nT;
                    sub_left = (SCHEME == SCHEME_SIMPLE) ? nT * nODE : 0;
                }
            }
            next += __popc(done);
        }
    }
}

}  // namespace cpab
