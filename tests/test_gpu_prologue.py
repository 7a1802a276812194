"""The prologue kernel (A = B theta and the per-cell expm, cpab_theta_to_trels)
on its three launch paths -- theta of 32 instances staged in shared memory
below the opt-in size, above it, and one thread per (instance, cell) for a d
too large to stage -- against the host: A = theta B^T (numpy, 1e-13
relative) and the oracle's expm of that A (2e-13 absolute on entries of
order 1: CUDA's exp and sin/cos against the host's libm, amplified by the
2D closed form where a random cell's linear block is nearly singular).
Each path sums over d in
order, so the three give the same A bit for bit on the same columns."""
import numpy as np
import pytest
import torch

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.cpa_space import CpaSpace

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _run(sp, B, theta, dt, sign):
    N, d = theta.shape
    D = B.shape[0]
    Bg = torch.as_tensor(B, device=DEV).contiguous()
    th = torch.as_tensor(theta, device=DEV).contiguous()
    A = torch.empty((N, D), dtype=torch.float64, device=DEV)
    sA, Tr = torch.empty_like(A), torch.empty_like(A)
    c = sp._ctx
    c.check(c.lib.cpab_theta_to_trels(c.h, _lib.ptr(Bg), d, _lib.ptr(th), N, dt, sign, _lib.ptr(A), _lib.ptr(sA),
                                      _lib.ptr(Tr), _lib.stream_ptr()))
    torch.cuda.synchronize()
    return A.cpu().numpy(), sA.cpu().numpy(), Tr.cpu().numpy()


@pytest.mark.parametrize("dim,nCs", [(1, (7,)), (2, (2, 2))])
@pytest.mark.parametrize("d", [40, 300, 700])      # 32 d doubles: 10 KB, 75 KB (opt-in), 175 KB (per-cell path)
@pytest.mark.parametrize("N", [1, 37, 100])
def test_theta_to_trels_paths_match_host(oracle_mod, dim, nCs, d, N):
    O = oracle_mod
    sp = CpaSpace([0.0] * dim, [1.0] * dim, nCs, tess="II" if dim == 1 else "I", device=DEV)
    ne = dim * (dim + 1)
    D = sp.nC * ne
    rng = np.random.default_rng(d + N)
    B = rng.standard_normal((D, d)) / np.sqrt(d)
    theta = rng.standard_normal((N, d))
    A, sA, Tr = _run(sp, B, theta, 0.02, -1)
    A_host = theta @ B.T
    np.testing.assert_allclose(A, A_host, rtol=1e-13, atol=1e-14)
    np.testing.assert_array_equal(sA, -A)
    sA_o, Tr_o = O.expm_cells(dim, A, 0.02, -1)
    np.testing.assert_array_equal(sA_o, sA)
    np.testing.assert_allclose(Tr, Tr_o, rtol=1e-13, atol=2e-13)


def test_theta_to_trels_same_sum_on_every_path():
    """The same B and theta padded to a d past each path's limit give the
    same A where the padding is zero (each path sums the columns in order)."""
    sp = CpaSpace([0.0], [1.0], (5,), tess="II", device=DEV)
    rng = np.random.default_rng(3)
    B = rng.standard_normal((10, 40))
    theta = rng.standard_normal((33, 40))
    outs = []
    for d in (40, 300, 700):
        Bp = np.zeros((10, d))
        Bp[:, :40] = B
        tp = np.zeros((33, d))
        tp[:, :40] = theta
        outs.append(_run(sp, Bp, tp, 0.02, 1)[0])
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])
