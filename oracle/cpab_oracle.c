/*
 * cpab_oracle.c -- CPU restatement of the CPAB transform hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library in cpabdiffeo_b200/csrc.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it; the product path never does.
 *
 * Every routine restates one routine of freifeld/cpabDiffeo (paths relative
 * to that project) in plain C.  Floating-point expressions keep the
 * reference's association order term by term because the cell lookup decides
 * branches by exact comparisons: a single differently-rounded operation moves
 * a point between the "Trel fast step" and the "midpoint fallback" paths.
 * Build with -ffp-contract=off (no fused multiply-add) -- see oracle/Makefile.
 *
 * Pinned against: the .npz fixtures in tests/golden, produced by the reference's own kernel
 * sources compiled as host code (oracle/ref_shim.cpp, tests/golden/make_golden.py).
 *
 * Conventions
 *   tess: 1 = type I (triangles / 5 tetrahedra per box), 2 = type II (boxes),
 *         the reference's TESS_TYPE macro (cpab/gpu/Calcs.py:159-162).
 *   A   : per cell, row-major DIM x (DIM+1) affine velocity matrix
 *         ("As_vectorized", cpab/cpaNd/_CpaCalcs.py:126-128).
 *   pts : row-major [nPts, DIM] ("C"-contiguous, cpab/gpu/Calcs.py:940-945).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

typedef struct {
    int dim;          /* 1, 2 or 3 */
    int tess;         /* 1 = I, 2 = II */
    int nC0, nC1, nC2;
    double inc_x, inc_y, inc_z;
} oracle_tess;

/* ------------------------------------------------------------------ */
/* cell lookup                                                          */
/* ------------------------------------------------------------------ */

/* mymin of cpab/gpu/calc_2Dto2D.cu:20-22: a if b >= a (or b is NaN), else
 * round(b). */
static inline int clamp_round_hi(int a, double b)
{
    return !(b < (double)a) ? a : (int)round(b);
}

/* round(min(n-1, max(0, (p - fmod(p, inc)) / inc))) -- the type-II box
 * coordinate along one axis: cpab/gpu/calc_1Dto1D.cu:64 (1D),
 * calc_2Dto2D.cu:46-47, calc_3Dto3D.cu:51-53.  The constant argument comes
 * first in fmin/fmax, which makes them agree with CUDA's min/max for NaN. */
static inline double box_coord(double p, int n, double inc)
{
    double q = (p - fmod(p, inc)) / inc;
    return round(fmin((double)(n - 1), fmax(0.0, q)));
}

/* cpab/gpu/calc_2Dto2D.cu:38-153, tess I branch (triangles 0 top, 1 right,
 * 2 bottom, 3 left inside each box; special rules outside the domain). */
static int cell_idx_2d_tri(const double *p, int nC0, int nC1, double inc_x, double inc_y)
{
    double p0 = fmin((nC0 * inc_x - 0.0000000001), fmax(0.0, p[0]));
    double p1 = fmin((nC1 * inc_y - 0.0000000001), fmax(0.0, p[1]));
    double xmod = fmod(p0, inc_x);
    double ymod = fmod(p1, inc_y);
    double x = xmod / inc_x;
    double y = ymod / inc_y;
    int c = clamp_round_hi(nC0 - 1, (p0 - xmod) / inc_x)
          + clamp_round_hi(nC1 - 1, (p1 - ymod) / inc_y) * nC0;
    c *= 4;
    if (p[0] <= 0) {                                       /* left of the domain */
        if (p[1] <= 0 && p[1] / inc_y < p[0] / inc_x) {
            /* triangle 0 */
        } else if (p[1] >= nC1 * inc_y && p[1] / inc_y - nC1 > -p[0] / inc_x) {
            c += 2;
        } else {
            c += 3;
        }
        return c;
    }
    if (p[0] >= nC0 * inc_x) {                             /* right of the domain */
        if (p[1] <= 0 && -p[1] / inc_y > p[0] / inc_x - nC0) {
            /* triangle 0 */
        } else if (p[1] >= nC1 * inc_y && p[1] / inc_y - nC1 > p[0] / inc_x - nC0) {
            c += 2;
        } else {
            c += 1;
        }
        return c;
    }
    if (p[1] <= 0) return c;                               /* above */
    if (p[1] >= nC1 * inc_y) return c + 2;                 /* below */
    if (x < y) {
        if (1 - x < y) c += 2; else c += 3;
    } else if (1 - x < y) {
        c += 1;
    }
    return c;
}

/* cpab/gpu/calc_3Dto3D.cu:43-137, tess I branch (5 tetrahedra per box with a
 * checkerboard flip).  The z clamp uses nC2*inc_x exactly as the reference
 * does (calc_3Dto3D.cu:59). */
static int cell_idx_3d_tet(const double *p, int nC0, int nC1, int nC2,
                           double inc_x, double inc_y, double inc_z)
{
    double p0 = fmin((nC0 * inc_x - 0.0000000001), fmax(0.0, p[0]));
    double p1 = fmin((nC1 * inc_y - 0.0000000001), fmax(0.0, p[1]));
    double p2 = fmin((nC2 * inc_x - 0.0000000001), fmax(0.0, p[2]));
    double xmod = fmod(p0, inc_x);
    double ymod = fmod(p1, inc_y);
    double zmod = fmod(p2, inc_z);
    int i = clamp_round_hi(nC0 - 1, ((p0 - xmod) / inc_x));
    int j = clamp_round_hi(nC1 - 1, ((p1 - ymod) / inc_y));
    int k = clamp_round_hi(nC2 - 1, ((p2 - zmod) / inc_z));
    int c = (i + j * nC0 + k * nC1 * nC0) * 5;
    double x = xmod / inc_x;
    double y = ymod / inc_y;
    double z = zmod / inc_z;
    int flip;
    if (k % 2 == 0)
        flip = (i % 2 == 0 && j % 2 == 1) || (i % 2 == 1 && j % 2 == 0);
    else
        flip = (i % 2 == 0 && j % 2 == 0) || (i % 2 == 1 && j % 2 == 1);
    if (flip) {
        double tmp = x;
        x = y;
        y = 1 - tmp;
    }
    if (-x - y + z >= 0)          c += 1;
    else if (x + y + z - 2 >= 0)  c += 2;
    else if (-x + y - z >= 0)     c += 3;
    else if (x - y - z >= 0)      c += 4;
    return c;
}

int oracle_cell_idx(const oracle_tess *t, const double *p)
{
    switch (t->dim) {
    case 1:
        return (int)box_coord(p[0], t->nC0, t->inc_x);
    case 2:
        if (t->tess == 2)
            return (int)(box_coord(p[0], t->nC0, t->inc_x)
                         + box_coord(p[1], t->nC1, t->inc_y) * t->nC0);
        return cell_idx_2d_tri(p, t->nC0, t->nC1, t->inc_x, t->inc_y);
    case 3:
        if (t->tess == 2)
            return (int)(box_coord(p[0], t->nC0, t->inc_x)
                         + box_coord(p[1], t->nC1, t->inc_y) * t->nC0
                         + box_coord(p[2], t->nC2, t->inc_z) * t->nC1 * t->nC0);
        return cell_idx_3d_tet(p, t->nC0, t->nC1, t->nC2, t->inc_x, t->inc_y, t->inc_z);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* affine velocity                                                      */
/* ------------------------------------------------------------------ */

/* A_times_b_affine, cpab/gpu/calc_1Dto1D.cu:18-34: x = A [b; 1] with the
 * sum taken left to right. */
static inline void affine_apply(int dim, double *x, const double *A, const double *b)
{
    if (dim == 1) {
        x[0] = A[0] * b[0] + A[1];
    } else if (dim == 2) {
        x[0] = A[0] * b[0] + A[1] * b[1] + A[2];
        x[1] = A[3] * b[0] + A[4] * b[1] + A[5];
    } else {
        x[0] = A[0] * b[0] + A[1] * b[1] + A[2] * b[2] + A[3];
        x[1] = A[4] * b[0] + A[5] * b[1] + A[6] * b[2] + A[7];
        x[2] = A[8] * b[0] + A[9] * b[1] + A[10] * b[2] + A[11];
    }
}

/* solveODE, cpab/gpu/calc_2Dto2D.cu:167-197 (1D/3D twins identical): explicit
 * midpoint, the cell is looked up at p only. Returns nothing; p in place. */
static void midpoint_solve(const oracle_tess *t, double *p, const double *As,
                           double h, int nSteps)
{
    const int dim = t->dim, ne = dim * (dim + 1);
    double v[3], pm[3];
    for (int s = 0; s < nSteps; ++s) {
        int c = oracle_cell_idx(t, p);
        const double *A = As + (size_t)c * ne;
        affine_apply(dim, v, A, p);
        for (int i = 0; i < dim; ++i) pm[i] = p[i] + h * v[i] / 2.;
        affine_apply(dim, v, A, pm);
        for (int i = 0; i < dim; ++i) p[i] += v[i] * h;
    }
}

/* calc_cell_idx kernel, cpab/gpu/calc_2Dto2D.cu:323-344. */
void oracle_calc_cell_idx(const oracle_tess *t, const double *pts, int32_t *out, int64_t n)
{
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        out[i] = oracle_cell_idx(t, pts + i * t->dim);
}

/* calc_v kernel, cpab/gpu/calc_2Dto2D.cu:561-602. */
void oracle_calc_v(const oracle_tess *t, const double *As, const double *pts,
                   double *out, int64_t n)
{
    const int dim = t->dim, ne = dim * (dim + 1);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double *p = pts + i * dim;
        int c = oracle_cell_idx(t, p);
        double v[3];
        affine_apply(dim, v, As + (size_t)c * ne, p);
        for (int k = 0; k < dim; ++k) out[i * dim + k] = v[k];
    }
}

/* One point of calc_T, cpab/gpu/calc_2Dto2D.cu:373-407.  Returns the number
 * of steps that took the midpoint fallback. */
static int integrate_point(const oracle_tess *t, const double *Trels, const double *As,
                           double *p, double dt, int nTimeSteps, int nStepsODE,
                           double *traj, int64_t stride)
{
    const int dim = t->dim, ne = dim * (dim + 1);
    double h = dt / (double)nStepsODE;
    double pn[3];
    int nfb = 0;
    for (int s = 0; s < nTimeSteps; ++s) {
        int c = oracle_cell_idx(t, p);
        affine_apply(dim, pn, Trels + (size_t)c * ne, p);
        int cn = oracle_cell_idx(t, pn);
        if (cn == c) {
            for (int i = 0; i < dim; ++i) p[i] = pn[i];
        } else {
            midpoint_solve(t, p, As, h, nStepsODE);
            ++nfb;
        }
        if (traj)
            for (int i = 0; i < dim; ++i) traj[(int64_t)s * stride + i] = p[i];
    }
    return nfb;
}

/* calc_T kernel (REF mode): Trels = expm(dt * sign * A), As = sign * A. */
int64_t oracle_calc_T(const oracle_tess *t, const double *Trels, const double *As,
                      const double *pts, double *out, int64_t n, double dt,
                      int nTimeSteps, int nStepsODE)
{
    const int dim = t->dim;
    int64_t nfb = 0;
    #pragma omp parallel for schedule(dynamic, 256) reduction(+:nfb)
    for (int64_t i = 0; i < n; ++i) {
        double p[3];
        for (int k = 0; k < dim; ++k) p[k] = pts[i * dim + k];
        nfb += integrate_point(t, Trels, As, p, dt, nTimeSteps, nStepsODE, NULL, 0);
        for (int k = 0; k < dim; ++k) out[i * dim + k] = p[k];
    }
    return nfb;
}

/* calc_T_simple kernel, cpab/gpu/calc_2Dto2D.cu:412-445: nTimeSteps*nStepsODE
 * midpoint steps of size dt/nStepsODE. */
void oracle_calc_T_simple(const oracle_tess *t, const double *As, const double *pts,
                          double *out, int64_t n, double dt, int nTimeSteps, int nStepsODE)
{
    const int dim = t->dim;
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        double p[3];
        for (int k = 0; k < dim; ++k) p[k] = pts[i * dim + k];
        midpoint_solve(t, p, As, dt / (double)nStepsODE, nStepsODE * nTimeSteps);
        for (int k = 0; k < dim; ++k) out[i * dim + k] = p[k];
    }
}

/* calc_trajectory, cpab/gpu/calc_2Dto2D.cu:499-556 plus the host-side
 * vstack of the initial points (cpab/cpaNd/_CpaCalcs.py:866-868):
 * traj is [(nTimeSteps+1), n, dim]. */
void oracle_calc_trajectory(const oracle_tess *t, const double *Trels, const double *As,
                            const double *pts, double *traj, int64_t n, double dt,
                            int nTimeSteps, int nStepsODE)
{
    const int dim = t->dim;
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        double p[3];
        for (int k = 0; k < dim; ++k) {
            p[k] = pts[i * dim + k];
            traj[i * dim + k] = p[k];
        }
        integrate_point(t, Trels, As, p, dt, nTimeSteps, nStepsODE,
                        traj + (n + i) * dim, n * dim);
    }
}

/* ------------------------------------------------------------------ */
/* per-cell affine exponentials                                         */
/* ------------------------------------------------------------------ */

/* 1D closed form, cpab/cpaNd/_CpaCalcs.py:285-292:
 * T = [exp(a dt), b dt (exp(a dt) - 1) / (a dt)], or [1, b dt] if a == 0. */
static void expm_1d(const double *sAdt, double *T)
{
    double a = sAdt[0], b = sAdt[1];
    T[0] = exp(a);
    T[1] = b;
    if (a != 0) T[1] = T[1] * (T[0] - 1) / a;
}

/* expm_2x2, cpab/gpu/expm/expm_affine_by_series_2D.py:28-74. */
static void expm_2x2(const double *A, double *E)
{
    double a = A[0], b = A[1], c = A[2], d = A[3];
    double disc = (a - d) * (a - d) + 4 * b * c;
    double e = exp((a + d) / 2);
    if (disc == 0) {
        E[0] = (1 + (a - d) / 2) * e;
        E[1] = b * e;
        E[2] = c * e;
        E[3] = (1 - (a - d) / 2) * e;
    } else if (disc > 0) {
        double delta = sqrt(disc) / 2;
        double ch = cosh(delta), sh = sinh(delta);
        double s = sh / delta;
        E[0] = (ch + (a - d) / 2 * s) * e;
        E[1] = b * s * e;
        E[2] = c * s * e;
        E[3] = (ch - (a - d) / 2 * s) * e;
    } else {
        double delta = sqrt(-disc) / 2;
        double co = cos(delta), si = sin(delta);
        double s = si / delta;
        E[0] = (co + (a - d) / 2 * s) * e;
        E[1] = b * s * e;
        E[2] = c * s * e;
        E[3] = (co - (a - d) / 2 * s) * e;
    }
}

/* Truncated Taylor series I + sum_{k=1..p} A^k / k! of an affine matrix
 * whose last homogeneous row is zero; A^k = A * A^(k-1).
 * cpab/gpu/expm/expm_affine_by_series_2D.py:156-232 (2D, p=12) and
 * expm_affine_by_series_3D.py:26-220 (3D). */
static void expm_taylor(int dim, const double *A, double *T, int p)
{
    const int nc = dim + 1, ne = dim * nc;
    double An[12], Bn[12];
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < nc; ++c)
            T[r * nc + c] = (r == c) ? 1.0 : 0.0;
    for (int k = 0; k < ne; ++k) { An[k] = A[k]; T[k] += An[k]; }
    if (p == 1) return;
    int fact = 1;
    for (int i = 2; i <= p; ++i) {
        memcpy(Bn, An, sizeof(double) * ne);
        fact *= i;
        for (int r = 0; r < dim; ++r)
            for (int c = 0; c < nc; ++c) {
                double acc = A[r * nc + 0] * Bn[0 * nc + c];
                for (int m = 1; m < dim; ++m) acc += A[r * nc + m] * Bn[m * nc + c];
                An[r * nc + c] = acc;
            }
        for (int k = 0; k < ne; ++k) T[k] += An[k] / fact;
    }
}

/* 2D affine expm, cpab/gpu/expm/expm_affine_by_series_2D.py:85-154: closed
 * form when the linear block is invertible, Taylor p=12 otherwise. */
static void expm_2d(const double *A, double *T)
{
    double A00 = A[0], A01 = A[1], A02 = A[2], A10 = A[3], A11 = A[4], A12 = A[5];
    double det = A00 * A11 - A01 * A10;
    if (det != 0) {
        double L[4] = {A00, A01, A10, A11}, E[4];
        expm_2x2(L, E);
        T[0] = E[0]; T[1] = E[1]; T[3] = E[2]; T[4] = E[3];
        double i00 = A11 / det, i11 = A00 / det, i01 = -A01 / det, i10 = -A10 / det;
        double a = i00 * A02 + i01 * A12;
        double b = i10 * A02 + i11 * A12;
        T[2] = (T[0] - 1) * a + (T[1]) * b;
        T[5] = (T[3]) * a + (T[4] - 1) * b;
        return;
    }
    expm_taylor(2, A, T, 12);
}

/* Per-cell Trel = expm(sign * dt * A) for N cells, following the host
 * preparation of cpab/cpaNd/_CpaCalcs.py:243-256 (sign first, then * dt)
 * and the dimension dispatch of :272-327.  signedA receives sign * A. */
void oracle_expm_cells(int dim, const double *A, int64_t N, double dt, int sign,
                       double *signedA, double *Trels)
{
    const int ne = dim * (dim + 1);
    #pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        double sA[12], sAdt[12];
        for (int k = 0; k < ne; ++k) {
            sA[k] = (sign < 0) ? -A[c * ne + k] : A[c * ne + k];
            sAdt[k] = sA[k] * dt;
            if (signedA) signedA[c * ne + k] = sA[k];
        }
        double *T = Trels + c * ne;
        if (dim == 1) expm_1d(sAdt, T);
        else if (dim == 2) expm_2d(sAdt, T);
        else expm_taylor(3, sAdt, T, 12);
    }
}

/* ------------------------------------------------------------------ */
/* exact 1D integration (ClosedFormInt)                                 */
/* ------------------------------------------------------------------ */

/* Restatement of cpab/cpa1d/calcs/ClosedFormInt.py for a zero-boundary 1D
 * space on [0,1] with nC equal intervals.  As: [nC, 2] (a, b) with v = a x + b
 * (sign already applied), x_tess: nC+1 vertices, velTess: velocity at each
 * vertex.  Returns 0 on success, 1 if the point exceeds nC crossings
 * (the reference raises ValueError, :155-160). */
static inline int cf_cell(double x, int nC)                    /* :23-27 */
{
    int i = (int)floor(x * nC);
    if (i < 0) i = 0;
    if (i > nC - 1) i = nC - 1;
    return i;
}
static inline double cf_v(const double *As, double x, int c)  /* :29-55 (scalar) */
{
    if (!(0 <= x && x <= 1)) return 0;
    return As[2 * c] * x + As[2 * c + 1];
}
static inline int allclose0(double v) { return fabs(v) <= 1e-8; } /* np.allclose(v,0) */

/* find_crossing_time, :193-256.  *next = -1 encodes "None". */
static double cf_crossing_time(const double *As, const double *x_tess, int nC,
                               double x, int c, int *next)
{
    double a = As[2 * c], b = As[2 * c + 1];
    double v = cf_v(As, x, c);
    *next = -1;
    if (allclose0(v)) return INFINITY;
    int cn = c + (v > 0 ? 1 : (v < 0 ? -1 : 0));
    if (!(0 <= cn && cn < nC)) return INFINITY;
    double xn;
    if (v > 0) { xn = x_tess[cn]; xn += 1e-16; }
    else       { xn = x_tess[c];  xn -= 1e-16; }
    double vn = cf_v(As, xn, cn);
    if (allclose0(vn)) return INFINITY;
    if ((v > 0) != (vn > 0) || (v < 0) != (vn < 0)) return INFINITY;
    double tt;
    if (xn == 0 || xn == 1) tt = INFINITY;
    else if (allclose0(a)) tt = (xn - x) / b;
    else tt = 1.0 / a * log((xn + b / a) / (x + b / a));
    *next = cn;
    return tt;
}

/* calc_affine_phi, :171-192. */
static double cf_affine_phi(const double *As, int c, double x, double tt)
{
    double a = As[2 * c], b = As[2 * c + 1];
    if (!(0 <= x && x <= 1)) { a = 0; b = 0; }
    if (a == 0) return x + tt * b;
    return exp(tt * a) * x + b * (exp(tt * a) - 1) / a;
}

/* calc_phi, :64-165. */
int oracle_closed_form_1d_point(const double *As, const double *x_tess, const double *velTess,
                                int nC, double x, double t, double *out)
{
    double x_old = x, x_new = x;
    double t_rem = t;
    int counter = 0;
    if (0 < x_old && x_old < 1) {
        for (int k = 0; k <= nC; ++k) {
            if (x_tess[k] == x_old) {
                if (!(velTess[k] > 0)) x_old = x_old - 1e-16;
                break;
            }
        }
    }
    for (;;) {
        int c = cf_cell(x_old, nC), cn;
        double tc = cf_crossing_time(As, x_tess, nC, x_old, c, &cn);
        int crossed;
        if (tc >= t_rem) { tc = t_rem; crossed = 0; }
        else crossed = 1;
        if (crossed) {
            if (cn > c) { x_new = x_tess[cn]; x_new += 1e-12; }
            else        { x_new = x_tess[c];  x_new -= 1e-12; }
        } else {
            x_new = cf_affine_phi(As, c, x_old, tc);
        }
        x_new = fmin(1.0, fmax(0.0, x_new));
        t_rem -= tc;
        if (!crossed) break;
        counter += 1;
        if (counter >= nC) { *out = x_new; return 1; }
        x_old = x_new;
    }
    *out = x_new;
    return 0;
}

int64_t oracle_closed_form_1d(const double *As, const double *x_tess, const double *velTess,
                              int nC, const double *pts, double *out, int64_t n, double t)
{
    int64_t nfail = 0;
    #pragma omp parallel for schedule(dynamic, 256) reduction(+:nfail)
    for (int64_t i = 0; i < n; ++i)
        nfail += oracle_closed_form_1d_point(As, x_tess, velTess, nC, pts[i], t, out + i);
    return nfail;
}

/* ------------------------------------------------------------------ */
/* bilinear remap and the Gaussian log-likelihood                       */
/* ------------------------------------------------------------------ */

/* Bilinear sample with cv2.remap conventions (x = column, y = row, integer
 * coordinates at pixel centres, taps outside the image read 0), the
 * semantics documented at cpab/cpa2d/TransformWrapper.py:286-317.  Map points
 * become pixel coordinates px = x*sx + ox, py = y*sy + oy: (W, -0.5, H, -0.5)
 * for points of the unit square with pixel centres at (i+0.5)/W, (1, 0, 1, 0)
 * for the reference's pixel-unit domain. */
static inline double tap(const float *img, int H, int W, int r, int c)
{
    return (r >= 0 && r < H && c >= 0 && c < W) ? (double)img[(int64_t)r * W + c] : 0.0;
}
static inline double bilinear(const float *img, int H, int W, double px, double py)
{
    double fx0 = floor(px), fy0 = floor(py);
    if (!(fx0 > -2.0 && fx0 < (double)W + 1.0 && fy0 > -2.0 && fy0 < (double)H + 1.0))
        return 0.0;
    double fx = px - fx0, fy = py - fy0;
    int c0 = (int)fx0, r0 = (int)fy0;
    double top = (1 - fx) * tap(img, H, W, r0, c0) + fx * tap(img, H, W, r0, c0 + 1);
    double bot = (1 - fx) * tap(img, H, W, r0 + 1, c0) + fx * tap(img, H, W, r0 + 1, c0 + 1);
    return (1 - fy) * top + fy * bot;
}

void oracle_remap(const double *map, const float *src, double *out, int H, int W,
                  double sx, double ox, double sy, double oy)
{
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)H * W; ++i)
        out[i] = bilinear(src, H, W, map[2 * i] * sx + ox, map[2 * i + 1] * sy + oy);
}

/* Gaussian log-likelihood of the warped source against dst:
 * sum_i -0.5 * (warped_i - dst_i)^2 / sigma^2, per
 * cpab/cpa2d/model/transformations/register/gpu/gaussian.py:15-34 and the
 * sum of _ScaleDependentLogLikelihoodGeneral.py:108-131.  Summed with
 * Kahan compensation in a fixed order. */
double oracle_remap_ssd(const double *map, const float *src, const float *dst, int H, int W,
                        double sx, double ox, double sy, double oy, double sigma, double *warped)
{
    double s = 0, comp = 0;
    double k = -0.5 / (sigma * sigma);
    for (int64_t i = 0; i < (int64_t)H * W; ++i) {
        double w = bilinear(src, H, W, map[2 * i] * sx + ox, map[2 * i + 1] * sy + oy);
        if (warped) warped[i] = w;
        double e = w - (double)dst[i];
        double term = e * e * k;
        double y = term - comp;
        double tt = s + y;
        comp = (tt - s) - y;
        s = tt;
    }
    return s;
}

/* ------------------------------------------------------------------ */
/* trilinear remap (3D) and its Gaussian log-likelihood                 */
/* ------------------------------------------------------------------ */

/* The 3D counterpart of bilinear() for remap3d (external of.gpu.remap,
 * called at cpab/cpa3d/TransformWrapper.py:254-286): a volume img [H, W, D]
 * indexed img[row][col][slice] -- the order of the reference's dense 3D grid,
 * np.mgrid[0:Ny, 0:Nx, 0:Nz] raveled with z fastest
 * (cpab/cpa3d/calcs/_CpaCalcs.py:45-76) -- is sampled at a point (x, y, z) =
 * (column, row, slice) in voxel coordinates, integer coordinates at voxel
 * centres, taps outside the volume read 0.  Interpolation along x, then y,
 * then z. */
static inline double tap3(const float *img, int H, int W, int D, int r, int c, int k)
{
    return (r >= 0 && r < H && c >= 0 && c < W && k >= 0 && k < D) ? (double)img[((int64_t)r * W + c) * D + k] : 0.0;
}
static inline double trilinear(const float *img, int H, int W, int D, double px, double py, double pz)
{
    double fx0 = floor(px), fy0 = floor(py), fz0 = floor(pz);
    if (!(fx0 > -2.0 && fx0 < (double)W + 1.0 && fy0 > -2.0 && fy0 < (double)H + 1.0 && fz0 > -2.0 &&
          fz0 < (double)D + 1.0))
        return 0.0;
    double fx = px - fx0, fy = py - fy0, fz = pz - fz0;
    int c0 = (int)fx0, r0 = (int)fy0, k0 = (int)fz0;
    double v[2];
    for (int dk = 0; dk < 2; ++dk) {
        double top = (1 - fx) * tap3(img, H, W, D, r0, c0, k0 + dk) + fx * tap3(img, H, W, D, r0, c0 + 1, k0 + dk);
        double bot = (1 - fx) * tap3(img, H, W, D, r0 + 1, c0, k0 + dk) +
                     fx * tap3(img, H, W, D, r0 + 1, c0 + 1, k0 + dk);
        v[dk] = (1 - fy) * top + fy * bot;
    }
    return (1 - fz) * v[0] + fz * v[1];
}

/* map [H*W*D, 3] (x, y, z); voxel coordinates px = x*sx + ox etc. */
void oracle_remap3d(const double *map, const float *src, double *out, int H, int W, int D, double sx, double ox,
                    double sy, double oy, double sz, double oz)
{
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)H * W * D; ++i)
        out[i] = trilinear(src, H, W, D, map[3 * i] * sx + ox, map[3 * i + 1] * sy + oy, map[3 * i + 2] * sz + oz);
}

double oracle_remap3d_ssd(const double *map, const float *src, const float *dst, int H, int W, int D, double sx,
                          double ox, double sy, double oy, double sz, double oz, double sigma, double *warped)
{
    double s = 0, comp = 0;
    double k = -0.5 / (sigma * sigma);
    for (int64_t i = 0; i < (int64_t)H * W * D; ++i) {
        double w = trilinear(src, H, W, D, map[3 * i] * sx + ox, map[3 * i + 1] * sy + oy, map[3 * i + 2] * sz + oz);
        if (warped) warped[i] = w;
        double e = w - (double)dst[i];
        double term = e * e * k;
        double y = term - comp;
        double tt = s + y;
        comp = (tt - s) - y;
        s = tt;
    }
    return s;
}
