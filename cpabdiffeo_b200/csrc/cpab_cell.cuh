// cpab_cell.cuh -- cell lookup and affine evaluation shared by every kernel.
//
// Two arithmetic families:
//
//  * exact (double): reproduces the reference's double-precision cell lookup
//    bit for bit (cpab/gpu/calc_1Dto1D.cu:56-259, calc_2Dto2D.cu:38-153,
//    calc_3Dto3D.cu:43-137) and its left-to-right affine sums with every
//    product and sum rounded on its own (no fused multiply-add).  The
//    reference evaluates  (p - fmod(p, inc)) / inc  and rounds it; this file
//    computes the same integer k and the same remainder r = fmod(p, inc)
//    without fmod or a division:
//        k = floor(p * (1/inc))            (estimate, off by at most one)
//        r = fma(-k, inc, p)               (exact: p - k*inc is representable
//                                           whenever k is the true quotient)
//        fix k by one if r < 0 or r >= inc, recompute r.
//    Because fmod is exact in IEEE arithmetic, r equals fmod(p, inc) bit for
//    bit, and round((p - r)/inc) equals k for every k < 2^50.  Quotients
//    that feed a comparison (xmod/inc) still use a correctly rounded
//    division, or an exact product when inc is a power of two.
//
//  * fast (float): the same tessellation geometry in single precision with
//    fused multiply-adds, for the FP32 mode, whose results are held to a
//    tolerance against the double-precision oracle.
//
// Everything is __host__ __device__ so the exact family can be checked
// against the oracle on the CPU (tests/test_cell_lookup_host.py).
#pragma once

#include <stdint.h>
#include <math.h>

#ifdef __CUDACC__
#define CPAB_HD __host__ __device__ __forceinline__
#else
#define CPAB_HD inline
#endif

// Non-contracted double arithmetic.  nvcc never fuses the __d*_rn
// intrinsics; the host build uses -ffp-contract=off.
#if defined(__CUDA_ARCH__)
#define XMUL(a, b) __dmul_rn((a), (b))
#define XADD(a, b) __dadd_rn((a), (b))
#define XSUB(a, b) __dsub_rn((a), (b))
#define XDIV(a, b) __ddiv_rn((a), (b))
#define XFMA(a, b, c) __fma_rn((a), (b), (c))
#else
#define XMUL(a, b) ((a) * (b))
#define XADD(a, b) ((a) + (b))
#define XSUB(a, b) ((a) - (b))
#define XDIV(a, b) ((a) / (b))
#define XFMA(a, b, c) fma((a), (b), (c))
#endif

namespace cpab {

// Geometry of one tessellation, precomputed on the host once per space.
// All derived doubles are formed exactly as the reference forms them
// (e.g. hi = (double)nC * inc - 1e-10, calc_2Dto2D.cu:55).
struct Tess {
    int dim;           // 1, 2, 3
    int tess;          // 1 = type I (simplices), 2 = type II (boxes)
    int nC0, nC1, nC2; // boxes per axis
    int nC;            // number of cells
    double inc[3];     // box size per axis (reference "incs")
    double inv_inc[3]; // 1/inc, used only as a quotient estimate
    double span[3];    // (double)nCk * inc_k
    double hi[3];      // clamp for type I: (double)nCk*inc_k - 1e-10 (axis 2 uses inc_x)
    int pow2[3];       // inc_k is a power of two: xmod/inc == xmod*(1/inc) exactly
    float finc[3], finv_inc[3], fspan[3], fhi[3];
};

// Geometry of a tessellation from box counts and box sizes, derived
// exactly as the reference derives its constants.  Returns false if the
// arguments are invalid.
inline bool make_tess(int dim, int tess, const int *nCs, const double *incs, Tess &t)
{
    t = Tess();
    if (dim < 1 || dim > 3 || (tess != 1 && tess != 2)) return false;
    t.dim = dim;
    t.tess = tess;
    int n[3] = {1, 1, 1};
    for (int k = 0; k < dim; ++k) {
        if (nCs[k] < 1 || !(incs[k] > 0) || !(incs[k] < INFINITY)) return false;
        n[k] = nCs[k];
    }
    t.nC0 = n[0];
    t.nC1 = dim > 1 ? n[1] : 0;
    t.nC2 = dim > 2 ? n[2] : 0;
    long long nC = (long long)n[0] * n[1] * n[2];
    if (tess == 1) nC *= (dim == 2 ? 4 : 5);
    if (nC > (1 << 20)) return false;
    t.nC = (int)nC;
    for (int k = 0; k < 3; ++k) {
        double inc = k < dim ? incs[k] : 1.0;
        t.inc[k] = inc;
        t.inv_inc[k] = 1.0 / inc;
        int e = 0;
        t.pow2[k] = (frexp(inc, &e) == 0.5) ? 1 : 0;
        t.span[k] = (double)n[k] * inc;
        t.hi[k] = (double)n[k] * inc - 0.0000000001;
    }
    // calc_3Dto3D.cu:59 clamps z with nC2*inc_x
    if (dim == 3 && tess == 1) t.hi[2] = (double)n[2] * t.inc[0] - 0.0000000001;
    for (int k = 0; k < 3; ++k) {
        t.finc[k] = (float)t.inc[k];
        t.finv_inc[k] = (float)(1.0 / t.inc[k]);
        t.fspan[k] = (float)t.span[k];
        double top = (dim == 3 && tess == 1 && k == 2) ? (double)n[2] * t.inc[0] : t.span[k];
        // float clamp strictly below the span so floor() stays in the last box
        t.fhi[k] = nextafterf((float)top, 0.0f);
    }
    return true;
}

// ---------------------------------------------------------------- exact

// k = trunc-toward-floor(p/inc) and r = fmod(p, inc) for finite p >= 0.
CPAB_HD void exact_floor_rem(double p, double inc, double inv, double &k, double &r)
{
    k = floor(p * inv);
    r = XFMA(-k, inc, p);
    if (r < 0.0) {
        k -= 1.0;
        r = XFMA(-k, inc, p);
    } else if (r >= inc) {
        k += 1.0;
        r = XFMA(-k, inc, p);
    }
}

// round(min(n-1, max(0, (p - fmod(p,inc))/inc)))  (type II / 1D axis).
// NaN and +-inf give 0 as in the reference (fmod(inf) is NaN, max(0,NaN)=0).
CPAB_HD int exact_box_coord(double p, int n, double inc, double inv)
{
    if (!(p >= 0.0) || !(p < INFINITY)) return 0;
    double k, r;
    exact_floor_rem(p, inc, inv, k, r);
    double lim = (double)(n - 1);
    return (int)(k < lim ? k : lim);
}

CPAB_HD double exact_frac(double xmod, double inc, double inv, int pow2)
{
    return pow2 ? XMUL(xmod, inv) : XDIV(xmod, inc);
}

// 2D type I (calc_2Dto2D.cu:53-148): 4 triangles per box, 0 top, 1 right,
// 2 bottom, 3 left; separate rules for points outside the domain.
CPAB_HD int exact_cell_2d_tri(const Tess &t, const double *p)
{
    const double ix = t.inc[0], iy = t.inc[1];
    double p0 = fmin(t.hi[0], fmax(0.0, p[0]));
    double p1 = fmin(t.hi[1], fmax(0.0, p[1]));
    double kx, xmod, ky, ymod;
    exact_floor_rem(p0, ix, t.inv_inc[0], kx, xmod);
    exact_floor_rem(p1, iy, t.inv_inc[1], ky, ymod);
    const double limx = (double)(t.nC0 - 1), limy = (double)(t.nC1 - 1);
    int c = ((int)(kx < limx ? kx : limx) + (int)(ky < limy ? ky : limy) * t.nC0) * 4;
    if (p[0] <= 0) {
        if (p[1] <= 0 && XDIV(p[1], iy) < XDIV(p[0], ix)) return c;
        if (p[1] >= t.span[1] && XSUB(XDIV(p[1], iy), (double)t.nC1) > XDIV(-p[0], ix)) return c + 2;
        return c + 3;
    }
    if (p[0] >= t.span[0]) {
        if (p[1] <= 0 && XDIV(-p[1], iy) > XSUB(XDIV(p[0], ix), (double)t.nC0)) return c;
        if (p[1] >= t.span[1] &&
            XSUB(XDIV(p[1], iy), (double)t.nC1) > XSUB(XDIV(p[0], ix), (double)t.nC0)) return c + 2;
        return c + 1;
    }
    if (p[1] <= 0) return c;
    if (p[1] >= t.span[1]) return c + 2;
    double x = exact_frac(xmod, ix, t.inv_inc[0], t.pow2[0]);
    double y = exact_frac(ymod, iy, t.inv_inc[1], t.pow2[1]);
    double omx = XSUB(1.0, x);
    if (x < y) return c + ((omx < y) ? 2 : 3);
    return c + ((omx < y) ? 1 : 0);
}

// 3D type I (calc_3Dto3D.cu:55-133): 5 tetrahedra per box with a
// checkerboard flip; the z clamp uses nC2*inc_x (hi[2] carries it).
CPAB_HD int exact_cell_3d_tet(const Tess &t, const double *p)
{
    double p0 = fmin(t.hi[0], fmax(0.0, p[0]));
    double p1 = fmin(t.hi[1], fmax(0.0, p[1]));
    double p2 = fmin(t.hi[2], fmax(0.0, p[2]));
    double ki, xmod, kj, ymod, kk, zmod;
    exact_floor_rem(p0, t.inc[0], t.inv_inc[0], ki, xmod);
    exact_floor_rem(p1, t.inc[1], t.inv_inc[1], kj, ymod);
    exact_floor_rem(p2, t.inc[2], t.inv_inc[2], kk, zmod);
    const double li = (double)(t.nC0 - 1), lj = (double)(t.nC1 - 1), lk = (double)(t.nC2 - 1);
    int i = (int)(ki < li ? ki : li), j = (int)(kj < lj ? kj : lj), k = (int)(kk < lk ? kk : lk);
    int c = (i + j * t.nC0 + k * t.nC1 * t.nC0) * 5;
    double x = exact_frac(xmod, t.inc[0], t.inv_inc[0], t.pow2[0]);
    double y = exact_frac(ymod, t.inc[1], t.inv_inc[1], t.pow2[1]);
    double z = exact_frac(zmod, t.inc[2], t.inv_inc[2], t.pow2[2]);
    bool flip = ((i ^ j ^ k) & 1) != 0;  // k even: i,j of different parity; k odd: same parity
    if (flip) {
        double tmp = x;
        x = y;
        y = XSUB(1.0, tmp);
    }
    if (XADD(XSUB(-x, y), z) >= 0) return c + 1;
    if (XSUB(XADD(XADD(x, y), z), 2.0) >= 0) return c + 2;
    if (XSUB(XADD(-x, y), z) >= 0) return c + 3;
    if (XSUB(XSUB(x, y), z) >= 0) return c + 4;
    return c;
}

template <int DIM, int TESS>
CPAB_HD int exact_cell(const Tess &t, const double *p)
{
    if (DIM == 1) return exact_box_coord(p[0], t.nC0, t.inc[0], t.inv_inc[0]);
    if (DIM == 2) {
        if (TESS == 2)
            return exact_box_coord(p[0], t.nC0, t.inc[0], t.inv_inc[0]) +
                   exact_box_coord(p[1], t.nC1, t.inc[1], t.inv_inc[1]) * t.nC0;
        return exact_cell_2d_tri(t, p);
    }
    if (TESS == 2)
        return exact_box_coord(p[0], t.nC0, t.inc[0], t.inv_inc[0]) +
               exact_box_coord(p[1], t.nC1, t.inc[1], t.inv_inc[1]) * t.nC0 +
               exact_box_coord(p[2], t.nC2, t.inc[2], t.inv_inc[2]) * t.nC1 * t.nC0;
    return exact_cell_3d_tet(t, p);
}

// x = A [b; 1], sums left to right, every operation rounded on its own
// (A_times_b_affine, calc_1Dto1D.cu:18-34).
template <int DIM>
CPAB_HD void exact_affine(double *x, const double *A, const double *b)
{
    if (DIM == 1) {
        x[0] = XADD(XMUL(A[0], b[0]), A[1]);
    } else if (DIM == 2) {
        x[0] = XADD(XADD(XMUL(A[0], b[0]), XMUL(A[1], b[1])), A[2]);
        x[1] = XADD(XADD(XMUL(A[3], b[0]), XMUL(A[4], b[1])), A[5]);
    } else {
        x[0] = XADD(XADD(XADD(XMUL(A[0], b[0]), XMUL(A[1], b[1])), XMUL(A[2], b[2])), A[3]);
        x[1] = XADD(XADD(XADD(XMUL(A[4], b[0]), XMUL(A[5], b[1])), XMUL(A[6], b[2])), A[7]);
        x[2] = XADD(XADD(XADD(XMUL(A[8], b[0]), XMUL(A[9], b[1])), XMUL(A[10], b[2])), A[11]);
    }
}

// One explicit-midpoint sub-step of solveODE (calc_2Dto2D.cu:177-196):
// pMid = p + h*v/2 ; p += vMid*h, with the cell of p for both evaluations.
template <int DIM>
CPAB_HD void exact_midpoint(double *p, const double *A, double h)
{
    double v[DIM], pm[DIM];
    exact_affine<DIM>(v, A, p);
#pragma unroll
    for (int i = 0; i < DIM; ++i) pm[i] = XADD(p[i], XDIV(XMUL(h, v[i]), 2.0));
    exact_affine<DIM>(v, A, pm);
#pragma unroll
    for (int i = 0; i < DIM; ++i) p[i] = XADD(p[i], XMUL(v[i], h));
}

// ---------------------------------------------------------------- fast (float)

CPAB_HD int fast_box_coord(float p, int n, float inv)
{
#ifdef __CUDA_ARCH__
    // one float->int conversion rounding down; NaN converts to 0, +-inf saturate
    int k = __float2int_rd(p * inv);
    return min(max(k, 0), n - 1);
#else
    float k = floorf(p * inv);
    k = fminf(fmaxf(k, 0.0f), (float)(n - 1));  // NaN -> 0
    return (int)k;
#endif
}

CPAB_HD int fast_cell_2d_tri(const Tess &t, const float *p)
{
    if (p[0] > 0.0f && p[0] < t.fhi[0] && p[1] > 0.0f && p[1] < t.fhi[1]) {
        // strictly inside the domain (the common case): the clamps below are
        // no-ops and none of the boundary rules applies -- same result
#ifdef __CUDA_ARCH__
        // both axes as one pair (FMUL2 / FADD2, each lane rounded as its scalar twin)
        const float2 uw = __fmul2_rn(make_float2(p[0], p[1]), make_float2(t.finv_inc[0], t.finv_inc[1]));
        const float kx = floorf(uw.x), ky = floorf(uw.y);
        const float2 xy = __fadd2_rn(uw, make_float2(-kx, -ky));
        const float x = xy.x, y = xy.y;
#else
        const float u = p[0] * t.finv_inc[0], w = p[1] * t.finv_inc[1];
        const float kx = floorf(u), ky = floorf(w);
        const float x = u - kx, y = w - ky;
#endif
        const int c = ((int)fminf(kx, (float)(t.nC0 - 1)) + (int)fminf(ky, (float)(t.nC1 - 1)) * t.nC0) * 4;
        const float omx = 1.0f - x;
        return c + ((x < y) ? ((omx < y) ? 2 : 3) : ((omx < y) ? 1 : 0));
    }
    float p0 = fminf(t.fhi[0], fmaxf(0.0f, p[0]));
    float p1 = fminf(t.fhi[1], fmaxf(0.0f, p[1]));
    float u = p0 * t.finv_inc[0], w = p1 * t.finv_inc[1];
    float kx = floorf(u), ky = floorf(w);
    float x = u - kx, y = w - ky;
    int c = ((int)fminf(kx, (float)(t.nC0 - 1)) + (int)fminf(ky, (float)(t.nC1 - 1)) * t.nC0) * 4;
    if (p[0] <= 0) {
        float a = p[0] * t.finv_inc[0], b = p[1] * t.finv_inc[1];
        if (p[1] <= 0 && b < a) return c;
        if (p[1] >= t.fspan[1] && b - (float)t.nC1 > -a) return c + 2;
        return c + 3;
    }
    if (p[0] >= t.fspan[0]) {
        float a = p[0] * t.finv_inc[0], b = p[1] * t.finv_inc[1];
        if (p[1] <= 0 && -b > a - (float)t.nC0) return c;
        if (p[1] >= t.fspan[1] && b - (float)t.nC1 > a - (float)t.nC0) return c + 2;
        return c + 1;
    }
    if (p[1] <= 0) return c;
    if (p[1] >= t.fspan[1]) return c + 2;
    float omx = 1.0f - x;
    if (x < y) return c + ((omx < y) ? 2 : 3);
    return c + ((omx < y) ? 1 : 0);
}

CPAB_HD int fast_cell_3d_tet(const Tess &t, const float *p)
{
    float u0 = fminf(t.fhi[0], fmaxf(0.0f, p[0])) * t.finv_inc[0];
    float u1 = fminf(t.fhi[1], fmaxf(0.0f, p[1])) * t.finv_inc[1];
    float u2 = fminf(t.fhi[2], fmaxf(0.0f, p[2])) * t.finv_inc[2];
    float fi = floorf(u0), fj = floorf(u1), fk = floorf(u2);
    float x = u0 - fi, y = u1 - fj, z = u2 - fk;
    int i = (int)fminf(fi, (float)(t.nC0 - 1));
    int j = (int)fminf(fj, (float)(t.nC1 - 1));
    int k = (int)fminf(fk, (float)(t.nC2 - 1));
    int c = (i + j * t.nC0 + k * t.nC1 * t.nC0) * 5;
    if ((i ^ j ^ k) & 1) {
        float tmp = x;
        x = y;
        y = 1.0f - tmp;
    }
    if (-x - y + z >= 0) return c + 1;
    if (x + y + z - 2.0f >= 0) return c + 2;
    if (-x + y - z >= 0) return c + 3;
    if (x - y - z >= 0) return c + 4;
    return c;
}

template <int DIM, int TESS>
CPAB_HD int fast_cell(const Tess &t, const float *p)
{
    if (DIM == 1) return fast_box_coord(p[0], t.nC0, t.finv_inc[0]);
    if (DIM == 2) {
        if (TESS == 2)
            return fast_box_coord(p[0], t.nC0, t.finv_inc[0]) +
                   fast_box_coord(p[1], t.nC1, t.finv_inc[1]) * t.nC0;
        return fast_cell_2d_tri(t, p);
    }
    if (TESS == 2)
        return fast_box_coord(p[0], t.nC0, t.finv_inc[0]) +
               fast_box_coord(p[1], t.nC1, t.finv_inc[1]) * t.nC0 +
               fast_box_coord(p[2], t.nC2, t.finv_inc[2]) * t.nC1 * t.nC0;
    return fast_cell_3d_tet(t, p);
}

template <int DIM>
CPAB_HD void fast_affine(float *x, const float *A, const float *b)
{
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        float acc = A[r * (DIM + 1) + DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) acc = fmaf(A[r * (DIM + 1) + c], b[c], acc);
        x[r] = acc;
    }
}

}  // namespace cpab
