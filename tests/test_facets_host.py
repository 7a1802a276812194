"""cpab_tess_facets (host only, no device): the library's facet tables -- the
ones the 2D/3D exact scheme reads -- equal the oracle's, which derives them
from the cells of the space builder (pinned to the reference's Tessellation
classes).  CPU only."""
import ctypes as C

import numpy as np
import pytest

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.space import build_space


@pytest.mark.parametrize("dim,nCs,tess", [(2, (4, 4), "I"), (2, (4, 4), "II"), (2, (16, 8), "I"),
                                          (3, (4, 4, 4), "I"), (3, (2, 2, 2), "II"), (3, (3, 2, 4), "I")])
def test_library_facets_equal_oracle(oracle_mod, dim, nCs, tess):
    O = oracle_mod
    L = _lib.load()
    geo = build_space(dim, nCs, tess)
    n = (C.c_int * 3)(*(list(nCs) + [1] * (3 - dim)))
    inc = (C.c_double * 3)(*(list(geo.incs) + [1.0] * (3 - dim)))
    nF = C.c_int()
    assert L.cpab_tess_facets(dim, geo.tess_code, n, inc, None, None, C.byref(nF)) == 0
    F = np.empty((geo.nC, nF.value, dim + 1))
    nb = np.empty((geo.nC, nF.value), np.int32)
    assert L.cpab_tess_facets(dim, geo.tess_code, n, inc, F.ctypes.data, nb.ctypes.data, C.byref(nF)) == 0
    Fo, nbo = O.cell_facets(O.tess_struct(dim, geo.tess_code, geo.nCs, geo.incs), geo.cells)
    np.testing.assert_allclose(F, Fo, rtol=0, atol=1e-15)
    np.testing.assert_array_equal(nb, nbo)


def test_facets_reject_bad_tessellation():
    L = _lib.load()
    n = (C.c_int * 3)(4, 4, 1)
    inc = (C.c_double * 3)(0.25, 0.25, 1.0)
    assert L.cpab_tess_facets(1, 1, n, inc, None, None, None) == 1  # CPAB_BAD_ARG
    assert L.cpab_tess_facets(4, 2, n, inc, None, None, None) == 1  # CPAB_BAD_ARG
