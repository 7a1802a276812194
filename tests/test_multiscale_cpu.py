"""Coarse-to-fine propagation on the host (no GPU): every fine cell takes the
affine map of the coarse cell containing it, and theta_fine = B_fine^T A_fine
reproduces the coarse velocity field exactly (the fine tessellation is nested
in the coarse one, so the duplicated field is continuous on the fine one)."""
import numpy as np
import pytest

from cpabdiffeo_b200.multiscale import parent_cells
from cpabdiffeo_b200.space import build_space

CASES = [
    (1, (5,), "II"),
    (2, (2, 3), "II"),
    (2, (2, 2), "I"),
    (3, (1, 2, 1), "II"),
    (3, (2, 2, 2), "I"),     # nested too (the reference stops at 3D type I, _Multiscale.py:259-262)
]


def _velocity(geo, A, pts):
    """v(x) = A_c [x; 1] with c the cell containing x (first match)."""
    from cpabdiffeo_b200.multiscale import _inside
    dim = geo.dim
    c = np.argmax(_inside(geo.cells, pts, geo.tess), axis=1)
    Ac = A.reshape(geo.nC, dim, dim + 1)[c]
    return np.einsum("pij,pj->pi", Ac, np.concatenate([pts, np.ones((len(pts), 1))], 1))


@pytest.mark.parametrize("dim,base,tess", CASES)
def test_propagation_reproduces_the_coarse_field(dim, base, tess):
    lo, hi = (0.0,) * dim, (1.0,) * dim
    gc = build_space(dim, base, tess, lo, hi, (True,) * dim)
    gf = build_space(dim, tuple(2 * b for b in base), tess, lo, hi, (True,) * dim)
    par = parent_cells(gc, gf)
    assert par.shape == (gf.nC,) and par.min() >= 0 and par.max() < gc.nC
    rng = np.random.default_rng(0)
    th_c = rng.normal(size=gc.d)
    A_c = gc.B @ th_c
    ne = gc.lengthAvee
    A_f = A_c.reshape(gc.nC, ne)[par].reshape(-1)
    th_f = gf.B.T @ A_f
    np.testing.assert_allclose(gf.B @ th_f, A_f, atol=1e-10)      # A_f lies in the fine CPA space
    pts = rng.uniform(0.01, 0.99, size=(500, dim))
    np.testing.assert_allclose(_velocity(gf, gf.B @ th_f, pts), _velocity(gc, A_c, pts), atol=1e-10)


def test_every_fine_cell_has_one_parent_2d_type_I():
    gc = build_space(2, (4, 4), "I", (0.0, 0.0), (1.0, 1.0), (True, True))
    gf = build_space(2, (8, 8), "I", (0.0, 0.0), (1.0, 1.0), (True, True))
    par = parent_cells(gc, gf)
    # each coarse triangle is split into 4 fine triangles
    assert np.array_equal(np.bincount(par, minlength=gc.nC), np.full(gc.nC, 4))
