"""The CUDA-graph captured batched step (CpaSpace.capture_batched): a replay
equals the eager launches bit for bit, and keeps doing so when the graph's
theta buffer and points are refilled between replays."""
import numpy as np
import pytest
import torch

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
P = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)


def _eager(sp, theta, x, offs, scheme, sign=1):
    out = torch.empty_like(x)
    sp.calc_T_batched(sp.tables_from_theta(theta, P["dt"], sign), x, out, offsets=offs, scheme=scheme, **P)
    return out


@pytest.mark.parametrize("dim,nCs,tess,prec,scheme,ragged", [
    (1, (100,), "II", torch.float32, _lib.SCHEME_EXACT, True),
    (1, (100,), "II", torch.float64, _lib.SCHEME_EXACT, True),
    (2, (4, 4), "I", torch.float32, _lib.SCHEME_REF, False),
    (2, (4, 4), "I", torch.float64, _lib.SCHEME_REF, True),
])
def test_graph_replay_equals_eager(dim, nCs, tess, prec, scheme, ragged):
    sp = CpaSpace([0.0] * dim, [1.0] * dim, nCs, tess=tess, device=DEV, precision=prec)
    rng = np.random.default_rng(31)
    n = 57
    prior = Prior.create(sp.geo, 0.1, 1.0)
    if ragged:
        sizes = rng.integers(0, 900, size=n)
        sizes[3] = 0
        offs = torch.as_tensor(np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64), device=DEV)
        total = int(sizes.sum())
    else:
        offs, total = None, n * 500
    x = torch.as_tensor(rng.uniform(0, 1, size=(total, dim)), dtype=prec, device=DEV)
    out = torch.full_like(x, float("nan"))
    cnt = torch.zeros(_lib.CNT_N, dtype=torch.int64, device=DEV)
    step = sp.capture_batched(n, x, out, offsets=offs, scheme=scheme, counters=cnt, **P)
    for rep in range(3):
        theta = torch.as_tensor(prior.sample(n, rng), device=DEV)
        if rep == 2:
            x.copy_(torch.as_tensor(rng.uniform(0, 1, size=(total, dim)), dtype=prec))
        cnt.zero_()
        out.fill_(float("nan"))
        step(theta)
        got = out.clone()
        pts_done = cnt[_lib.CNT_POINTS].item()
        want = _eager(sp, theta, x, offs, scheme)
        torch.cuda.synchronize()
        assert torch.equal(got, want), rep
        assert pts_done == total
