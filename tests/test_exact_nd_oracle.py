"""The EXACT scheme's FP64 CPU oracle in 2D and 3D (oracle/cpab_oracle_exact.c):
boundary-hitting times by facet bracketing and Newton, the reference's
closed-form steps kept where the step stays in its cell.  The reference has
no 2D/3D hitting-time integrator, so the oracle is validated by properties:

  * it converges to the reference's own scheme as its midpoint sub-steps
    shrink (calc_T with nStepsODE = 10^4 agrees to ~1e-13);
  * on a field that moves x only, with the velocity of a 1D CPA field, its x
    coordinate is the 1D closed form (ClosedFormInt, pinned to the
    reference's calc_phi) and y does not move;
  * the inverse flow undoes the forward flow;
  * facet tables: every cell's vertices satisfy its own facets, and the
    neighbour relation is symmetric.
CPU only.
"""
import numpy as np
import pytest

from cpabdiffeo_b200.space import Prior, build_space

SPACES = [(2, (4, 4), "I"), (2, (4, 4), "II"), (3, (4, 4, 4), "I"), (3, (2, 2, 2), "II")]
DT, NT = 0.02, 50


def _setup(O, dim, nCs, tess):
    geo = build_space(dim, nCs, tess)
    t = O.tess_struct(dim, geo.tess_code, geo.nCs, geo.incs)
    F, nb = O.cell_facets(t, geo.cells)
    return geo, t, F, nb


@pytest.mark.parametrize("dim,nCs,tess", SPACES)
def test_facet_tables(oracle_mod, dim, nCs, tess):
    geo, t, F, nb = _setup(oracle_mod, dim, nCs, tess)
    for c in range(geo.nC):
        for v in geo.cells[c]:
            assert (F[c, :, :dim] @ v[:dim] + F[c, :, dim]).max() < 1e-15
        for k, n in enumerate(nb[c]):
            if n >= 0:
                assert c in nb[n]
    np.testing.assert_allclose(np.linalg.norm(F[:, :, :dim], axis=-1), 1.0, rtol=1e-15)
    # boundary facets: one per box side on the boundary (two triangles per box face in 3D type I)
    n_bdry = (nb < 0).sum()
    if dim == 2:
        side = 2 * (nCs[0] + nCs[1])
    else:
        side = 2 * (nCs[0] * nCs[1] + nCs[1] * nCs[2] + nCs[0] * nCs[2])
    assert n_bdry == side * (2 if (dim == 3 and tess == "I") else 1)


@pytest.mark.parametrize("dim,nCs,tess", SPACES)
def test_exact_converges_to_the_reference_scheme(oracle_mod, dim, nCs, tess):
    O = oracle_mod
    geo, t, F, nb = _setup(O, dim, nCs, tess)
    rng = np.random.default_rng(7)
    pr = Prior.create(geo, 0.1 if dim < 3 else 0.15, 1.0 if dim < 3 else 0.5)
    A = (geo.B @ pr.sample(1, rng)[0] * 2.0).reshape(geo.nC, -1)
    x = rng.uniform(0, 1, (1500, dim))
    sA, Tr = O.expm_cells(dim, A, DT, 1)
    ex, cnt = O.calc_T_exact(t, Tr, sA, F, nb, x, DT, NT, 100)
    assert cnt[2] > 100 and cnt[3] == 0          # crossings happened; no fallback
    ref_fine, _ = O.calc_T(t, Tr, sA, x, DT, NT, 10000)
    ref_100, _ = O.calc_T(t, Tr, sA, x, DT, NT, 100)
    e_fine = np.abs(ex - ref_fine).max()
    e_100 = np.abs(ex - ref_100).max()
    assert e_fine < 1e-10
    assert e_fine < e_100 / 100                   # the reference scheme approaches it as nStepsODE grows


@pytest.mark.parametrize("dim,nCs,tess", SPACES)
def test_exact_inverse_undoes_forward(oracle_mod, dim, nCs, tess):
    O = oracle_mod
    geo, t, F, nb = _setup(O, dim, nCs, tess)
    rng = np.random.default_rng(8)
    pr = Prior.create(geo, 0.1, 1.0)
    A = (geo.B @ pr.sample(1, rng)[0] * 2.0).reshape(geo.nC, -1)
    x = rng.uniform(0.02, 0.98, (1000, dim))
    sA, Tr = O.expm_cells(dim, A, DT, 1)
    sAi, Tri = O.expm_cells(dim, A, DT, -1)
    y, _ = O.calc_T_exact(t, Tr, sA, F, nb, x, DT, NT, 100)
    z, _ = O.calc_T_exact(t, Tri, sAi, F, nb, y, DT, NT, 100)
    assert np.abs(z - x).max() < 1e-9


@pytest.mark.parametrize("tess", ["I", "II"])
def test_exact_2d_reduces_to_the_1d_closed_form(oracle_mod, tess):
    O = oracle_mod
    g1 = build_space(1, (4,), "II")
    rng = np.random.default_rng(5)
    a1 = (g1.B @ Prior.create(g1, 0.3, 1.0).sample(1, rng)[0] * 3).reshape(4, 2)
    g2, t, F, nb = _setup(O, 2, (4, 4), tess)
    per = 4 if tess == "I" else 1
    A = np.zeros((g2.nC, 2, 3))
    for i in range(4):
        for j in range(4):
            cells = slice((j + 4 * i) * per, (j + 4 * i + 1) * per)
            A[cells, 0, 0], A[cells, 0, 2] = a1[j, 0], a1[j, 1]
    A = A.reshape(g2.nC, 6)
    x = rng.uniform(0, 1, (3000, 2))
    sA, Tr = O.expm_cells(2, A, DT, 1)
    ex, cnt = O.calc_T_exact(t, Tr, sA, F, nb, x, DT, NT, 100)
    cf, nf = O.closed_form_1d(a1, 4, x[:, 0], DT * NT)
    assert nf == 0 and cnt[2] > 1000
    assert np.abs(ex[:, 0] - cf).max() < 1e-10
    assert np.array_equal(ex[:, 1], x[:, 1])
