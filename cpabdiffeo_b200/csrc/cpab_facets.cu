// cpab_facets.cu -- host-side facet tables of a tessellation, for the EXACT
// scheme's boundary-hitting times in 2D/3D.
//
// Every cell is a convex polytope: a triangle (2D type I), a tetrahedron
// (3D type I) or a box (type II).  Its facets are stored as rows
// (n, -h) with n the outward unit normal and h the offset, so that
// g(x) = n . x - h <= 0 inside; nbr holds the cell across each facet, or -1
// on the domain boundary.  Cell and vertex order follow the reference's
// Tessellation classes (cpab/cpa2d/Tessellation.py:73-138,
// cpab/cpa3d/Tessellation.py:62-200): type I triangles (centre, ul, ur),
// (centre, ur, lr), (centre, lr, ll), (centre, ll, ul) per box; type I
// tetrahedra five per box with the checkerboard flip of odd boxes.
// Simplex facet k is opposite vertex k; box facets are (x_lo, x_hi, y_lo,
// y_hi, z_lo, z_hi).  The neighbour across a facet is the cell that the
// library's own lookup finds just outside the facet's centroid.
#include <cmath>
#include <vector>

#include "cpab_ctx.h"

namespace cpab {

namespace {

struct V3 {
    double x[3];
};

// vertices of every cell, in the reference's order
void cell_vertices(const Tess &t, const int *nCs, std::vector<std::vector<V3>> &cells)
{
    const double inc[3] = {t.inc[0], t.inc[1], t.inc[2]};
    auto P = [&](int j, int i, int k) {
        V3 v{{j * inc[0], i * inc[1], k * inc[2]}};
        return v;
    };
    cells.clear();
    if (t.dim == 1) {
        for (int j = 0; j < nCs[0]; ++j) cells.push_back({P(j, 0, 0), P(j + 1, 0, 0)});
    } else if (t.dim == 2) {
        for (int i = 0; i < nCs[1]; ++i)
            for (int j = 0; j < nCs[0]; ++j) {
                const V3 ul = P(j, i, 0), ur = P(j + 1, i, 0), ll = P(j, i + 1, 0), lr = P(j + 1, i + 1, 0);
                if (t.tess == 2) {
                    cells.push_back({ul, ur, lr, ll});
                } else {
                    const V3 ctr{{(j + 0.5) * inc[0], (i + 0.5) * inc[1], 0.0}};
                    cells.push_back({ctr, ul, ur});
                    cells.push_back({ctr, ur, lr});
                    cells.push_back({ctr, lr, ll});
                    cells.push_back({ctr, ll, ul});
                }
            }
    } else {
        for (int k = 0; k < nCs[2]; ++k)
            for (int i = 0; i < nCs[1]; ++i)
                for (int j = 0; j < nCs[0]; ++j) {
                    V3 ul0 = P(j, i, k), ur0 = P(j + 1, i, k), ll0 = P(j, i + 1, k), lr0 = P(j + 1, i + 1, k);
                    V3 ul1 = P(j, i, k + 1), ur1 = P(j + 1, i, k + 1), ll1 = P(j, i + 1, k + 1),
                       lr1 = P(j + 1, i + 1, k + 1);
                    if (t.tess == 2) {
                        cells.push_back({ul0, ur0, lr0, ll0, ul1, ur1, lr1, ll1});
                        continue;
                    }
                    if ((i + j + k) % 2 == 1) {
                        V3 a = ul0, b = ul1;
                        ul0 = ur0; ur0 = lr0; lr0 = ll0; ll0 = a;
                        ul1 = ur1; ur1 = lr1; lr1 = ll1; ll1 = b;
                    }
                    cells.push_back({ll1, ur1, ul0, lr0});
                    cells.push_back({ul1, ur1, ll1, ul0});
                    cells.push_back({lr1, ur1, ll1, lr0});
                    cells.push_back({ll0, ul0, lr0, ll1});
                    cells.push_back({ur0, ul0, lr0, ur1});
                }
    }
}

int lookup(const Tess &t, const double *p)
{
    if (t.dim == 1) return exact_cell<1, 2>(t, p);
    if (t.dim == 2) return t.tess == 1 ? exact_cell<2, 1>(t, p) : exact_cell<2, 2>(t, p);
    return t.tess == 1 ? exact_cell<3, 1>(t, p) : exact_cell<3, 2>(t, p);
}

}  // namespace

int facets_per_cell(const Tess &t) { return (t.tess == 1 && t.dim > 1) ? t.dim + 1 : 2 * t.dim; }

int build_facets(const Tess &t, const int *nCs, std::vector<double> &F, std::vector<int> &nbr)
{
    const int dim = t.dim, nh = dim + 1, nF = facets_per_cell(t);
    const bool simplex = t.tess == 1 && dim > 1;
    const double inc[3] = {t.inc[0], t.inc[1], t.inc[2]};
    double minc = inc[0], ext[3];
    for (int i = 0; i < dim; ++i) {
        minc = std::fmin(minc, inc[i]);
        ext[i] = nCs[i] * inc[i];
    }
    std::vector<std::vector<V3>> cells;
    cell_vertices(t, nCs, cells);
    const int nC = (int)cells.size();
    F.assign((size_t)nC * nF * nh, 0.0);
    nbr.assign((size_t)nC * nF, -1);
    for (int c = 0; c < nC; ++c) {
        const std::vector<V3> &V = cells[c];
        const int nV = (int)V.size();
        for (int k = 0; k < nF; ++k) {
            double n[3] = {0, 0, 0}, h = 0, m[3] = {0, 0, 0};
            if (simplex) {
                int idx[3] = {0, 0, 0}, q = 0;
                for (int j = 0; j <= dim; ++j)
                    if (j != k) idx[q++] = j;
                const double *a = V[idx[0]].x, *b = V[idx[1]].x;
                if (dim == 2) {
                    n[0] = b[1] - a[1];
                    n[1] = -(b[0] - a[0]);
                } else {
                    const double *cc = V[idx[2]].x;
                    double u[3], w[3];
                    for (int i = 0; i < 3; ++i) {
                        u[i] = b[i] - a[i];
                        w[i] = cc[i] - a[i];
                    }
                    n[0] = u[1] * w[2] - u[2] * w[1];
                    n[1] = u[2] * w[0] - u[0] * w[2];
                    n[2] = u[0] * w[1] - u[1] * w[0];
                }
                double nn = 0;
                for (int i = 0; i < dim; ++i) nn += n[i] * n[i];
                nn = std::sqrt(nn);
                for (int i = 0; i < dim; ++i) n[i] /= nn;
                for (int i = 0; i < dim; ++i) h += n[i] * a[i];
                double side = -h;
                for (int i = 0; i < dim; ++i) side += n[i] * V[k].x[i];
                if (side > 0) {
                    for (int i = 0; i < dim; ++i) n[i] = -n[i];
                    h = -h;
                }
                for (int j = 0; j < dim; ++j)
                    for (int i = 0; i < dim; ++i) m[i] += V[idx[j]].x[i] / dim;
            } else {
                const int ax = k / 2, upper = k % 2;
                double lo = V[0].x[ax], hi = V[0].x[ax];
                for (int j = 1; j < nV; ++j) {
                    lo = std::fmin(lo, V[j].x[ax]);
                    hi = std::fmax(hi, V[j].x[ax]);
                }
                n[ax] = upper ? 1.0 : -1.0;
                h = upper ? hi : -lo;
                for (int i = 0; i < dim; ++i) {
                    double s = 0;
                    for (int j = 0; j < nV; ++j) s += V[j].x[i];
                    m[i] = s / nV;
                }
                m[ax] = upper ? hi : lo;
            }
            double *row = &F[((size_t)c * nF + k) * nh];
            for (int i = 0; i < dim; ++i) row[i] = n[i];
            row[dim] = -h;
            double q[3] = {0, 0, 0};
            bool inside = true;
            for (int i = 0; i < dim; ++i) {
                q[i] = m[i] + 1e-7 * minc * n[i];
                if (!(q[i] > 0.0 && q[i] < ext[i])) inside = false;
            }
            const int nb = inside ? lookup(t, q) : -1;
            nbr[(size_t)c * nF + k] = (nb == c) ? -1 : nb;
        }
    }
    return nF;
}

}  // namespace cpab

using namespace cpab;

extern "C" int cpab_tess_facets(int dim, int tess, const int *nCs, const double *incs, double *facets, int *nbr,
                                int *n_facets_per_cell)
{
    if (dim < 1 || dim > 3 || (tess != 1 && tess != 2) || (dim == 1 && tess == 1) || !nCs || !incs)
        return fail(nullptr, CPAB_BAD_ARG, "invalid tessellation");
    Tess t;
    if (!make_tess(dim, tess, nCs, incs, t)) return fail(nullptr, CPAB_BAD_ARG, "invalid nCs/incs");
    const int nF = facets_per_cell(t);
    if (n_facets_per_cell) *n_facets_per_cell = nF;
    if (!facets && !nbr) return CPAB_OK;
    std::vector<double> F;
    std::vector<int> nb;
    build_facets(t, nCs, F, nb);
    if (facets) std::memcpy(facets, F.data(), F.size() * sizeof(double));
    if (nbr) std::memcpy(nbr, nb.data(), nb.size() * sizeof(int));
    return CPAB_OK;
}
