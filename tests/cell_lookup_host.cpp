// Host build of cpabdiffeo_b200/csrc/cpab_cell.cuh for tests/test_cell_lookup_host.py:
// the exact (double) lookup compiled with -ffp-contract=off, exported with C linkage.
#include "cpab_cell.cuh"

using namespace cpab;

extern "C" void host_exact_cells(const Tess *t, const double *pts, int *out, long n)
{
    for (long i = 0; i < n; ++i) {
        const double *p = pts + i * t->dim;
        int c;
        if (t->dim == 1) c = exact_cell<1, 2>(*t, p);
        else if (t->dim == 2) c = t->tess == 1 ? exact_cell<2, 1>(*t, p) : exact_cell<2, 2>(*t, p);
        else c = t->tess == 1 ? exact_cell<3, 1>(*t, p) : exact_cell<3, 2>(*t, p);
        out[i] = c;
    }
}

extern "C" void host_fast_cells(const Tess *t, const float *pts, int *out, long n)
{
    for (long i = 0; i < n; ++i) {
        const float *p = pts + i * t->dim;
        int c;
        if (t->dim == 1) c = fast_cell<1, 2>(*t, p);
        else if (t->dim == 2) c = t->tess == 1 ? fast_cell<2, 1>(*t, p) : fast_cell<2, 2>(*t, p);
        else c = t->tess == 1 ? fast_cell<3, 1>(*t, p) : fast_cell<3, 2>(*t, p);
        out[i] = c;
    }
}

extern "C" int host_tess_size() { return (int)sizeof(Tess); }

extern "C" int host_make_tess(int dim, int tess, const int *nCs, const double *incs, Tess *out)
{
    return make_tess(dim, tess, nCs, incs, *out) ? 1 : 0;
}
