"""The exact 1D kernel (k_exact1d, through cpab_calc_T with CPAB_SCHEME_EXACT)
against the output of the reference's own ClosedFormInt.calc_phi
(cpab/cpa1d/calcs/ClosedFormInt.py:64-165), run by
tests/golden/make_golden_py_ref.py: prior draws on 100, 20 and 5 cells,
forward and inverse, uniform points, every vertex and its 1e-17 / 1e-16 /
1e-12 neighbours, the domain ends and points outside.

Tolerances: FP64 1e-12 absolute (outputs lie in [0, 1]); FP32 storage
(the inputs rounded to float32 before the flow, the outputs rounded after
it) 1e-5 relative with a 1e-6 absolute floor for outputs near 0.
"""
from pathlib import Path

import numpy as np
import pytest
import torch

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.cpa_space import CpaSpace

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
PYREF = Path(__file__).resolve().parent / "golden" / "pyref"


def _cases():
    z = np.load(PYREF / "closedform_1d.npz")
    for i in range(len(z["nC"])):
        nC = int(z["nC"][i])
        A = z["A"][z["A_offsets"][i]:z["A_offsets"][i + 1]].reshape(nC, 2)
        sl = slice(z["offsets"][i], z["offsets"][i + 1])
        yield nC, A, z["x"][sl], z["out"][sl]


@pytest.mark.parametrize("precision", [torch.float64, torch.float32])
def test_exact_1d_kernel_matches_reference_calc_phi(precision):
    spaces = {}
    worst = 0.0
    for nC, A, x, ref in _cases():
        if nC not in spaces:
            spaces[nC] = CpaSpace([0.0], [1.0], (nC,), device=DEV, precision=precision)
        sp = spaces[nC]
        sA, Tr = sp.tables_from_A(torch.as_tensor(A.reshape(1, -1), device=DEV), 0.02, 1)
        xg = torch.as_tensor(x[:, None], dtype=precision, device=DEV)
        out = torch.full_like(xg, float("nan"))
        cnt = torch.zeros(_lib.CNT_N, dtype=torch.int64, device=DEV)
        c = sp._ctx
        c.check(c.lib.cpab_calc_T(c.h, _lib.ptr(sA[0]), _lib.ptr(Tr[0]), _lib.ptr(xg), _lib.ptr(out), x.size,
                                  _lib.CPAB_F64 if precision == torch.float64 else _lib.CPAB_F32,
                                  _lib.SCHEME_EXACT, 0.02, 50, 100, _lib.ptr(cnt), _lib.stream_ptr()))
        got = out.cpu().numpy().astype(np.float64)[:, 0]
        assert cnt[_lib.CNT_FAILED].item() == 0
        if precision == torch.float64:
            np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12)
        else:
            np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6)
        worst = max(worst, float(np.abs(got - ref).max()))
    print(f"max abs error vs the reference's calc_phi: {worst:.3e}")
