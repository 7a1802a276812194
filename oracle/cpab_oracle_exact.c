/*
 * cpab_oracle_exact.c -- FP64 CPU oracle of the EXACT integration scheme in
 * 2D and 3D (boundary-hitting times), written by this project.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the library's EXACT scheme; only
 * tests/ and bench.py's checking legs load it).
 *
 * The reference integrates in closed form across cell boundaries only in 1D
 * (cpab/cpa1d/calcs/ClosedFormInt.py:64-256).  In 2D/3D its calc_T
 * (cpab/gpu/calc_2Dto2D.cu:348-408) takes closed-form steps Trel =
 * expm(dt A_c) while a step's end stays in the start cell and otherwise
 * re-integrates the step with nStepsODE explicit-midpoint sub-steps
 * (calc_2Dto2D.cu:167-197).  The EXACT scheme keeps the closed-form step
 * and its keep test, and re-integrates a step that leaves its cell with
 * nStepsODE sub-steps of the exact flow, S_c = expm(h A_c), h = dt/nStepsODE:
 *
 *   a sub-step whose end stays in the cell is kept; one whose end leaves it
 *   brackets the exit.  Inside cell c the flow is x(t) = expm(t A_c)[p; 1];
 *   it leaves through an interior facet k (outward unit normal n_k, offset
 *   h_k: n_k . x <= h_k inside) at the first root of
 *   g_k(t) = n_k . x(t) - h_k.  For every interior facet the sub-step's end
 *   violates, a safeguarded Newton iteration (g_k' = n_k . v_c(x(t))) finds
 *   the root in [0, h]; the earliest is the exit time tau.  The point moves
 *   to x(tau), the cell becomes the facet's neighbour, and the rest of the
 *   sub-step (h - tau) is the neighbour's flow, exiting again if its end
 *   leaves that cell.  Facets on the domain boundary never exit (the
 *   velocity's normal component vanishes there).
 *
 * x(t) for arbitrary t is the action of the exponential on [p; 1] by its
 * Taylor series, x(t) = p + sum_k w_k with w_1 = t (L p + b),
 * w_k = (t / k) L w_{k-1} (A = [L | b]), until the terms fall below the
 * rounding of the sum (t <= h).
 *
 * Fallback: when no interior facet explains a sub-step's exit (a point on
 * the domain boundary) or more than 4 nC + 16 crossings occur in one
 * sub-step, the sub-step's end point is kept, as in the reference scheme.
 *
 * Counters: [0] closed-form steps kept, [1] steps with an exit,
 * [2] facet crossings, [3] fallbacks.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int dim;
    int tess;
    int nC0, nC1, nC2;
    double inc_x, inc_y, inc_z;
} oracle_tess;

int oracle_cell_idx(const oracle_tess *t, const double *p);

#define EX_MAX_NEWTON 100
#define EX_MAX_TAYLOR 60

static int n_cells(const oracle_tess *t)
{
    int n = t->nC0 * (t->dim > 1 ? t->nC1 : 1) * (t->dim > 2 ? t->nC2 : 1);
    if (t->tess == 1 && t->dim == 2) n *= 4;
    if (t->tess == 1 && t->dim == 3) n *= 5;
    return n;
}

/* Facets of every cell from its vertices cells[nC][nV][dim+1] (homogeneous):
 * facets[nC][nF][dim+1] = (n, -h) with n the outward unit normal, nbr[nC][nF]
 * the cell across the facet or -1 on the domain boundary.  Simplices (nV =
 * dim + 1): facet k is opposite vertex k.  Boxes (nV = 2^dim): facets
 * x_i >= lo_i, x_i <= hi_i in the order (lo_0, hi_0, lo_1, ...).
 * Returns nF. */
int oracle_cell_facets(const oracle_tess *t, const double *cells, int nV, double *facets, int *nbr)
{
    const int dim = t->dim, nh = dim + 1, nC = n_cells(t);
    const int simplex = (nV == dim + 1) && dim > 1;
    const int nF = simplex ? dim + 1 : 2 * dim;
    const double incs[3] = {t->inc_x, t->inc_y, t->inc_z};
    const int nCs[3] = {t->nC0, t->nC1, t->nC2};
    double minc = incs[0];
    for (int i = 1; i < dim; ++i) minc = fmin(minc, incs[i]);
    for (int c = 0; c < nC; ++c) {
        const double *V = cells + (size_t)c * nV * nh;
        for (int k = 0; k < nF; ++k) {
            double n[3] = {0, 0, 0}, h = 0, m[3] = {0, 0, 0};
            if (simplex) {
                int idx[3] = {0, 0, 0}, q = 0;
                for (int j = 0; j <= dim; ++j)
                    if (j != k) idx[q++] = j;
                const double *a = V + idx[0] * nh, *b = V + idx[1] * nh;
                if (dim == 2) {
                    n[0] = b[1] - a[1];
                    n[1] = -(b[0] - a[0]);
                } else {
                    const double *cc = V + idx[2] * nh;
                    double u[3], w[3];
                    for (int i = 0; i < 3; ++i) { u[i] = b[i] - a[i]; w[i] = cc[i] - a[i]; }
                    n[0] = u[1] * w[2] - u[2] * w[1];
                    n[1] = u[2] * w[0] - u[0] * w[2];
                    n[2] = u[0] * w[1] - u[1] * w[0];
                }
                double nn = 0;
                for (int i = 0; i < dim; ++i) nn += n[i] * n[i];
                nn = sqrt(nn);
                for (int i = 0; i < dim; ++i) n[i] /= nn;
                for (int i = 0; i < dim; ++i) h += n[i] * a[i];
                double side = -h;
                for (int i = 0; i < dim; ++i) side += n[i] * V[k * nh + i];
                if (side > 0) {  /* the opposite vertex must be inside */
                    for (int i = 0; i < dim; ++i) n[i] = -n[i];
                    h = -h;
                }
                for (int j = 0; j < dim; ++j)
                    for (int i = 0; i < dim; ++i) m[i] += V[idx[j] * nh + i] / dim;
            } else {
                const int ax = k / 2, upper = k % 2;
                double lo = V[ax], hi = V[ax];
                for (int j = 1; j < nV; ++j) {
                    lo = fmin(lo, V[j * nh + ax]);
                    hi = fmax(hi, V[j * nh + ax]);
                }
                n[ax] = upper ? 1.0 : -1.0;
                h = upper ? hi : -lo;
                for (int i = 0; i < dim; ++i) {
                    double s = 0;
                    for (int j = 0; j < nV; ++j) s += V[j * nh + i];
                    m[i] = s / nV;
                }
                m[ax] = upper ? hi : lo;
            }
            double *F = facets + ((size_t)c * nF + k) * nh;
            for (int i = 0; i < dim; ++i) F[i] = n[i];
            F[dim] = -h;
            /* neighbour: the cell of the facet centroid nudged outward */
            double q[3];
            int inside = 1;
            for (int i = 0; i < dim; ++i) {
                q[i] = m[i] + 1e-7 * minc * n[i];
                if (!(q[i] > 0.0 && q[i] < nCs[i] * incs[i])) inside = 0;
            }
            nbr[c * nF + k] = inside ? oracle_cell_idx(t, q) : -1;
            if (nbr[c * nF + k] == c) nbr[c * nF + k] = -1;
        }
    }
    return nF;
}

/* y = expm(t A)[p; 1] (spatial part) by the Taylor series of the action. */
static void expmv(int dim, const double *A, const double *p, double t, double *y)
{
    const int nh = dim + 1;
    double w[3], nw[3];
    for (int i = 0; i < dim; ++i) {
        double v = A[i * nh + dim];
        for (int j = 0; j < dim; ++j) v += A[i * nh + j] * p[j];
        w[i] = t * v;
        y[i] = p[i] + w[i];
    }
    for (int k = 2; k <= EX_MAX_TAYLOR; ++k) {
        double big = 0, ymax = 0;
        for (int i = 0; i < dim; ++i) {
            double s = 0;
            for (int j = 0; j < dim; ++j) s += A[i * nh + j] * w[j];
            nw[i] = s * (t / k);
        }
        for (int i = 0; i < dim; ++i) {
            w[i] = nw[i];
            y[i] += w[i];
            big = fmax(big, fabs(w[i]));
            ymax = fmax(ymax, fabs(y[i]));
        }
        if (big <= 1e-18 * (ymax + 1e-300)) break;
    }
}

static inline double facet_g(int dim, const double *F, const double *x)
{
    double g = F[dim];
    for (int i = 0; i < dim; ++i) g += F[i] * x[i];
    return g;
}

static inline double facet_dg(int dim, const double *F, const double *A, const double *x)
{
    const int nh = dim + 1;
    double d = 0;
    for (int i = 0; i < dim; ++i) {
        double v = A[i * nh + dim];
        for (int j = 0; j < dim; ++j) v += A[i * nh + j] * x[j];
        d += F[i] * v;
    }
    return d;
}

/* Root of g(t) = n . x(t) - h in [lo, hi], g(lo) <= 0 < g(hi). */
static double facet_root(int dim, const double *A, const double *F, const double *p, double lo, double hi,
                         double glo, double ghi)
{
    double y[3];
    double t = lo - glo * (hi - lo) / (ghi - glo);
    if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
    for (int it = 0; it < EX_MAX_NEWTON; ++it) {
        expmv(dim, A, p, t, y);
        const double g = facet_g(dim, F, y);
        if (g > 0) hi = t; else lo = t;
        if (g == 0) return t;
        const double dg = facet_dg(dim, F, A, y);
        double tn = t - g / dg;
        if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
        /* within about two ulps (4.5e-16 is at least two ulps in every binade) */
        if (fabs(tn - t) <= 4.5e-16 * fmax(fabs(t), 1e-300) || hi - lo <= 4.5e-16 * hi) return tn;
        t = tn;
    }
    return 0.5 * (lo + hi);
}

static inline void affine3(int dim, const double *A, const double *x, double *y)
{
    const int nh = dim + 1;
    for (int i = 0; i < dim; ++i) {
        double v = A[i * nh + dim];
        for (int j = 0; j < dim; ++j) v += A[i * nh + j] * x[j];
        y[i] = v;
    }
}

/* S = expm(h A) of a cell's affine matrix (homogeneous, bottom row 0), as
 * the DIM x (DIM+1) top block, by its Taylor series. */
static void expm_sub(int dim, const double *A, double h, double *S)
{
    const int nh = dim + 1;
    double P[12], Q[12];
    for (int i = 0; i < dim * nh; ++i) {
        P[i] = h * A[i];
        S[i] = P[i];
    }
    for (int k = 2; k <= EX_MAX_TAYLOR; ++k) {
        double big = 0;
        for (int i = 0; i < dim; ++i)
            for (int j = 0; j < nh; ++j) {
                double v = 0;
                for (int m = 0; m < dim; ++m) v += h * A[i * nh + m] * P[m * nh + j];
                Q[i * nh + j] = v / k;
            }
        for (int i = 0; i < dim * nh; ++i) {
            P[i] = Q[i];
            S[i] += P[i];
            big = fmax(big, fabs(P[i]));
        }
        if (big <= 1e-18) break;
    }
    for (int i = 0; i < dim; ++i) S[i * nh + i] += 1.0;
}

/* The exact flow over one sub-step of length h from p in cell c whose end
 * point (q, from the cell's sub-step map) left the cell: exit times through
 * interior facets, the neighbour across the exited facet, the rest of the
 * sub-step there (again exiting if its end leaves that cell).  p becomes the
 * point at the sub-step's end; returns its cell. */
static int exact_substep_crossing(const oracle_tess *t, const double *As, const double *facets, const int *nbr,
                                  int nF, int c, double *p, const double *q, double h, int cap, int64_t *cnt)
{
    const int dim = t->dim, nh = dim + 1, ne = dim * nh;
    double y[3];
    double s = h;
    memcpy(y, q, sizeof(double) * dim);
    for (int crossings = 0;; ) {
        if (oracle_cell_idx(t, y) == c) {
            memcpy(p, y, sizeof(double) * dim);
            return c;
        }
        const double *A = As + (size_t)c * ne;
        const double *Fc = facets + (size_t)c * nF * nh;
        const int *nb = nbr + c * nF;
        double tau = s;
        int kbest = -1;
        for (int k = 0; k < nF; ++k) {
            if (nb[k] < 0) continue;
            const double *F = Fc + k * nh;
            const double ghi = facet_g(dim, F, y);
            if (!(ghi > 0)) continue;
            const double glo = facet_g(dim, F, p);
            const double r = (glo >= 0) ? 0.0 : facet_root(dim, A, F, p, 0.0, s, glo, ghi);
            if (kbest < 0 || r < tau) {
                tau = r;
                kbest = k;
            }
        }
        if (kbest < 0 || !(tau == tau) || ++crossings > cap) {
            /* no interior facet explains the exit (or too many crossings):
             * keep the sub-step's end point, as the reference scheme does */
            memcpy(p, y, sizeof(double) * dim);
            ++cnt[3];
            return oracle_cell_idx(t, p);
        }
        double z[3];
        expmv(dim, A, p, tau, z);
        memcpy(p, z, sizeof(double) * dim);
        s -= tau;
        c = nb[kbest];
        ++cnt[2];
        if (!(s > 0)) return c;
        expmv(dim, As + (size_t)c * ne, p, s, y);
    }
}

static void exact_point(const oracle_tess *t, const double *Trels, const double *As, const double *Ss,
                        const double *facets, const int *nbr, int nF, double *p, double dt, int nT, int nODE,
                        int64_t *cnt)
{
    const int dim = t->dim, nh = dim + 1, ne = dim * nh;
    const int cap = 4 * n_cells(t) + 16;
    const double h = dt / (double)nODE;
    double q[3];
    for (int step = 0; step < nT; ++step) {
        int c = oracle_cell_idx(t, p);
        affine3(dim, Trels + (size_t)c * ne, p, q);
        if (oracle_cell_idx(t, q) == c) {  /* the reference's keep test */
            memcpy(p, q, sizeof(double) * dim);
            ++cnt[0];
            continue;
        }
        ++cnt[1];
        /* the step again in nStepsODE sub-steps of the exact flow; a sub-step
         * whose end leaves its cell is resolved at the exit times */
        for (int k = 0; k < nODE; ++k) {
            affine3(dim, Ss + (size_t)c * ne, p, q);
            if (oracle_cell_idx(t, q) == c) {
                memcpy(p, q, sizeof(double) * dim);
                continue;
            }
            c = exact_substep_crossing(t, As, facets, nbr, nF, c, p, q, h, cap, cnt);
        }
    }
}

/* EXACT calc_T: Trels = expm(dt * sign * A), As = sign * A; facets / nbr
 * from oracle_cell_facets.  counters[4] accumulated (may be NULL). */
void oracle_calc_T_exact(const oracle_tess *t, const double *Trels, const double *As, const double *facets,
                         const int *nbr, int nF, const double *pts, double *out, int64_t n, double dt,
                         int nTimeSteps, int nStepsODE, int64_t *counters)
{
    const int dim = t->dim, ne = dim * (dim + 1), nC = n_cells(t);
    double *Ss = (double *)malloc(sizeof(double) * (size_t)nC * ne);
    if (!Ss) return;
    for (int c = 0; c < nC; ++c) expm_sub(dim, As + (size_t)c * ne, dt / (double)nStepsODE, Ss + (size_t)c * ne);
    int64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    #pragma omp parallel for schedule(dynamic, 64) reduction(+:c0, c1, c2, c3)
    for (int64_t i = 0; i < n; ++i) {
        double p[3];
        int64_t cnt[4] = {0, 0, 0, 0};
        for (int k = 0; k < dim; ++k) p[k] = pts[i * dim + k];
        exact_point(t, Trels, As, Ss, facets, nbr, nF, p, dt, nTimeSteps, nStepsODE, cnt);
        for (int k = 0; k < dim; ++k) out[i * dim + k] = p[k];
        c0 += cnt[0]; c1 += cnt[1]; c2 += cnt[2]; c3 += cnt[3];
    }
    free(Ss);
    if (counters) {
        counters[0] += c0; counters[1] += c1; counters[2] += c2; counters[3] += c3;
    }
}
