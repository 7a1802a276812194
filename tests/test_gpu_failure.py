"""Failure handling without faulting the GPU: cancellation through the
context's flag (before a launch and from another host thread
during one), NaN inputs surfacing as a counter instead of a hang, and the
context staying usable afterwards."""
import threading
import time

import numpy as np
import pytest
import torch

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
P = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)


def _batch(n_theta, n_per, precision=torch.float32, seed=0):
    sp = CpaSpace([0.0], [1.0], (100,), device=DEV, precision=precision)
    rng = np.random.default_rng(seed)
    theta = torch.as_tensor(Prior.create(sp.geo, 0.1, 1.0).sample(n_theta, rng), device=DEV)
    x = torch.as_tensor(rng.uniform(0, 1, (n_theta * n_per, 1)), dtype=precision, device=DEV)
    return sp, theta, x


def _run(sp, theta, x, scheme=_lib.SCHEME_REF):
    tables = sp.tables_from_theta(theta, P["dt"], 1)
    out = torch.full_like(x, float("nan"))
    cnt = torch.zeros(_lib.CNT_N, dtype=torch.int64, device=DEV)
    sp.calc_T_batched(tables, x, out, scheme=scheme, counters=cnt, **P)
    return out, cnt


@pytest.mark.parametrize("scheme", [_lib.SCHEME_REF, _lib.SCHEME_EXACT])
def test_cancel_before_launch_then_clear(scheme):
    sp, theta, x = _batch(64, 4000)
    sp.cancel()
    out, cnt = _run(sp, theta, x, scheme)
    torch.cuda.synchronize()
    assert cnt[_lib.CNT_POINTS].item() == 0 and cnt[_lib.CNT_CANCELLED].item() > 0
    assert torch.isnan(out).all()
    sp.clear_cancel()
    out, cnt = _run(sp, theta, x, scheme)
    torch.cuda.synchronize()
    assert cnt[_lib.CNT_POINTS].item() == x.shape[0] and cnt[_lib.CNT_CANCELLED].item() == 0
    assert not torch.isnan(out).any()


def test_cancel_from_another_thread_mid_run():
    sp, theta, x = _batch(512, 40000)                       # ~20M points, tens of ms through the REF scheme
    full, _ = _run(sp, theta, x)
    torch.cuda.synchronize()
    t = threading.Timer(0.003, sp.cancel)
    t.start()
    out, cnt = _run(sp, theta, x)
    torch.cuda.synchronize()
    t.join()
    sp.clear_cancel()
    done = ~torch.isnan(out[:, 0])
    assert cnt[_lib.CNT_CANCELLED].item() > 0
    assert 0 <= done.sum().item() < x.shape[0]
    # the points that were finished are the right ones
    assert torch.equal(out[done], full[done])
    # and the context still works
    again, cnt2 = _run(sp, theta, x)
    torch.cuda.synchronize()
    assert torch.equal(again, full) and cnt2[_lib.CNT_POINTS].item() == x.shape[0]


@pytest.mark.parametrize("scheme", [_lib.SCHEME_REF, _lib.SCHEME_EXACT])
def test_nan_theta_is_counted_not_hung(scheme):
    sp, theta, x = _batch(4, 3000, torch.float64)
    theta[1, 3] = float("nan")
    t0 = time.perf_counter()
    out, cnt = _run(sp, theta, x, scheme)
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 30
    assert cnt[_lib.CNT_POINTS].item() == x.shape[0]
    nan_rows = torch.isnan(out[:, 0]).sum().item()
    assert cnt[_lib.CNT_NAN].item() == nan_rows
    if scheme == _lib.SCHEME_REF:
        # 1D zero boundary: the clamp maps NaN to NaN, so the poisoned instance is all NaN
        assert nan_rows == 3000
    assert not torch.isnan(out[:3000]).any() and not torch.isnan(out[6000:]).any()
