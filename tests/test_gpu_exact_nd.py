"""The EXACT scheme in 2D and 3D on the GPU (k_integrate<..., SCHEME_EXACT>,
through cpab_calc_T / cpab_calc_T_batched) against its FP64 CPU oracle
(oracle/cpab_oracle_exact.c, validated against the reference scheme as
nStepsODE -> 10^4 and against the 1D closed form).

Tolerances: FP64 1e-12 absolute (the two compute the same hitting times
with different but exact evaluations of the flow); FP32 points (FP64
hitting times) 1e-5 * max(1, |x|) against the FP64 oracle.  Counters: the
GPU resolves the same number of facet crossings as the oracle, up to a few
points whose crossing sits within rounding of a sub-step end.
"""
import numpy as np
import pytest
import torch

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
DT, NT, NODE = 0.02, 50, 100
SPACES = [(2, (4, 4), "I"), (2, (4, 4), "II"), (3, (4, 4, 4), "I"), (3, (2, 2, 2), "II")]


def _case(O, dim, nCs, tess, precision, seed, scale=2.0, n=4000):
    sp = CpaSpace([0.0] * dim, [1.0] * dim, nCs, tess=tess, device=DEV, precision=precision)
    rng = np.random.default_rng(seed)
    pr = Prior.create(sp.geo, 0.1 if dim < 3 else 0.15, 1.0 if dim < 3 else 0.5)
    theta = pr.sample(3, rng) * scale
    t = O.tess_struct(dim, sp.geo.tess_code, sp.geo.nCs, sp.geo.incs)
    F, nb = O.cell_facets(t, sp.geo.cells)
    x = rng.uniform(0, 1, (n, dim))
    return sp, theta, t, F, nb, x


@pytest.mark.parametrize("dim,nCs,tess", SPACES)
@pytest.mark.parametrize("precision", [torch.float64, torch.float32])
@pytest.mark.parametrize("sign", [1, -1])
def test_exact_nd_matches_oracle(oracle_mod, dim, nCs, tess, precision, sign):
    O = oracle_mod
    sp, theta, t, F, nb, x = _case(O, dim, nCs, tess, precision, 41 + dim)
    sA, Tr = sp.tables_from_theta(torch.as_tensor(theta, device=DEV), DT, sign)
    xg = torch.as_tensor(x, dtype=precision, device=DEV)
    xin = xg.double().cpu().numpy()
    prec = _lib.CPAB_F64 if precision == torch.float64 else _lib.CPAB_F32
    c = sp._ctx
    for i in range(theta.shape[0]):
        out = torch.full_like(xg, float("nan"))
        cnt = torch.zeros(_lib.CNT_N, dtype=torch.int64, device=DEV)
        c.check(c.lib.cpab_calc_T(c.h, _lib.ptr(sA[i]), _lib.ptr(Tr[i]), _lib.ptr(xg), _lib.ptr(out), x.shape[0],
                                  prec, _lib.SCHEME_EXACT, DT, NT, NODE, _lib.ptr(cnt), _lib.stream_ptr()))
        ref, ocnt = O.calc_T_exact(t, Tr[i].cpu().numpy(), sA[i].cpu().numpy(), F, nb, xin, DT, NT, NODE)
        got = out.cpu().numpy().astype(np.float64)
        cnt = cnt.cpu().numpy()
        assert cnt[_lib.CNT_POINTS] == x.shape[0]
        assert ocnt[2] > 50                                   # the flow crossed facets
        if precision == torch.float64:
            np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12)
            assert abs(int(cnt[_lib.CNT_CROSSINGS]) - int(ocnt[2])) <= max(3, ocnt[2] // 1000)
            assert cnt[_lib.CNT_FAILED] == ocnt[3]
        else:
            assert np.abs(got - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("dim,nCs,tess", [(2, (4, 4), "I"), (3, (4, 4, 4), "I")])
def test_exact_nd_batched_ragged_equals_single(oracle_mod, dim, nCs, tess):
    """A ragged batch (with an empty instance) equals the per-instance calls bit for bit."""
    sp, theta, t, F, nb, x = _case(oracle_mod, dim, nCs, tess, torch.float32, 5, n=3000)
    tables = sp.tables_from_theta(torch.as_tensor(theta, device=DEV), DT, 1)
    sizes = np.array([1700, 0, 1300])
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    xg = torch.as_tensor(x, dtype=torch.float32, device=DEV)
    out = torch.empty_like(xg)
    p = dict(dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    sp.calc_T_batched(tables, xg, out, offsets=torch.as_tensor(offs, device=DEV), scheme=_lib.SCHEME_EXACT, **p)
    c = sp._ctx
    for i in (0, 2):
        sl = slice(int(offs[i]), int(offs[i + 1]))
        one = torch.empty_like(xg[sl])
        c.check(c.lib.cpab_calc_T(c.h, _lib.ptr(tables[0][i]), _lib.ptr(tables[1][i]), _lib.ptr(xg[sl]),
                                  _lib.ptr(one), int(sizes[i]), _lib.CPAB_F32, _lib.SCHEME_EXACT, DT, NT, NODE,
                                  None, _lib.stream_ptr()))
        assert torch.equal(one, out[sl])


def test_exact_nd_more_accurate_than_reference_scheme(oracle_mod):
    """Against the reference scheme with 10^4 midpoint sub-steps per leaving
    step (the oracle's restatement of calc_T), the exact scheme's error is
    far below the reference scheme's at nStepsODE = 100."""
    O = oracle_mod
    sp, theta, t, F, nb, x = _case(O, 2, (4, 4), "I", torch.float64, 9, n=2000)
    sA, Tr = sp.tables_from_theta(torch.as_tensor(theta[:1], device=DEV), DT, 1)
    xg = torch.as_tensor(x, device=DEV)
    out_ex, out_ref = torch.empty_like(xg), torch.empty_like(xg)
    p = dict(dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    sp.calc_T_batched((sA, Tr), xg, out_ex, scheme=_lib.SCHEME_EXACT, **p)
    sp.calc_T_batched((sA, Tr), xg, out_ref, scheme=_lib.SCHEME_REF, **p)
    fine, _ = O.calc_T(t, Tr[0].cpu().numpy(), sA[0].cpu().numpy(), x, DT, NT, 10000)
    e_ex = np.abs(out_ex.cpu().numpy() - fine).max()
    e_ref = np.abs(out_ref.cpu().numpy() - fine).max()
    assert e_ex < 1e-9 and e_ex < e_ref / 100, (e_ex, e_ref)
