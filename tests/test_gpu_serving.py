"""Continuous-batching server: every result is the same alone and inside the
mix (bit-exact: the kernels are per point / per image with fixed reduction
order and per-job random streams), requests submitted while others run are
admitted, and a tight memory budget still drains the queue."""
import inspect

import numpy as np
import pytest
import torch
from scipy.ndimage import gaussian_filter

from cpabdiffeo_b200.serving import CpabServer, RegistrationRequest, TransformRequest
from cpabdiffeo_b200.space import Prior, build_space

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _mix(rng):
    reqs = []
    for i in range(12):
        kind = i % 4
        if kind == 0:
            dim, nCs, tess = 1, (int(rng.choice([16, 100])),), "II"
        elif kind == 1:
            dim, nCs, tess = 2, (4, 4), "I"
        elif kind == 2:
            dim, nCs, tess = 3, (2, 2, 2), "II"
        else:
            dim, nCs, tess = 2, (2, 2), "I"
        geo = build_space(dim, nCs, tess)
        theta = Prior.create(geo, 0.1, 1.0).sample(1, rng)[0]
        n = int(10 ** rng.uniform(2, 4))
        dt = np.float64 if i % 3 == 0 else np.float32
        reqs.append(TransformRequest(dim, nCs, theta, rng.uniform(0, 1, size=(n, dim)).astype(dt), tess=tess,
                                     sign=1 if i % 5 else -1))
    for j in range(2):
        H, W = 24 + 8 * j, 32
        src = gaussian_filter(rng.uniform(0, 1, (H, W)).astype(np.float32), 3.0)
        dst = np.roll(src, 1, axis=1) + rng.normal(0, 0.02, (H, W)).astype(np.float32)
        reqs.append(RegistrationRequest(src, dst, n_steps=30, seed=100 + j))
    return reqs


def _same(a, b):
    if isinstance(a, dict):
        return np.array_equal(a["theta"], b["theta"]) and a["ll"] == b["ll"] and a["accepted"] == b["accepted"]
    return np.array_equal(a, b)


@pytest.mark.parametrize("reserved", [False, True])
def test_alone_equals_in_mix(reserved):
    """reserved: the server's stream buffers, pinned pool and job image slots
    are allocated up front (CpabServer.reserve) and reused across requests."""
    rng = np.random.default_rng(0)
    reqs = _mix(rng)
    srv = CpabServer(device=DEV)
    if reserved:
        srv.reserve(dims=3, image_side=40)
    first, late = reqs[:8], reqs[8:]
    ids = [srv.submit(r) for r in first]
    srv.step()                                  # work is on the GPU ...
    ids += [srv.submit(r) for r in late]        # ... when the rest arrives
    srv.run_until_idle()
    assert len(srv.done) == len(reqs)
    for rid, r in zip(ids, reqs):
        alone = CpabServer(device=DEV)
        aid = alone.submit(r)
        alone.run_until_idle()
        assert _same(srv.done[rid].result, alone.done[aid].result), (rid, type(r).__name__)


def test_transform_results_match_oracle(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(1)
    geo = build_space(2, (4, 4), "I")
    theta = Prior.create(geo, 0.1, 1.0).sample(3, rng)
    reqs = [TransformRequest(2, (4, 4), theta[i], rng.uniform(0, 1, (500 + 300 * i, 2)), tess="I") for i in range(3)]
    srv = CpabServer(device=DEV)
    ids = [srv.submit(r) for r in reqs]
    srv.run_until_idle()
    sp = srv.space(2, (4, 4), "I", torch.float64)
    t = O.tess_struct(2, 1, (4, 4), geo.incs)
    for rid, r in zip(ids, reqs):
        sA, Tr = sp.tables_from_theta(torch.as_tensor(r.theta[None], device=DEV), 0.02, 1)
        ref, _ = O.calc_T(t, Tr[0].cpu().numpy(), sA[0].cpu().numpy(), r.pts, 0.02, 50, 100)
        np.testing.assert_array_equal(srv.done[rid].result, ref)


def test_memory_budget_admission_drains():
    rng = np.random.default_rng(2)
    geo = build_space(1, (100,), "II")
    theta = Prior.create(geo, 0.1, 1.0).sample(20, rng)
    srv = CpabServer(device=DEV, memory_budget_bytes=200_000)   # about one request at a time
    ids = [srv.submit(TransformRequest(1, (100,), theta[i], rng.uniform(0, 1, (8000, 1)).astype(np.float32)))
           for i in range(20)]
    peak = 0
    while not srv.idle():
        srv.step()
        peak = max(peak, srv.in_use)
    assert len(srv.done) == 20 and srv.in_use == 0
    assert peak <= 200_000 + 2 * 8000 * 4 + (1 << 16)
    lat = srv.latencies()
    assert (lat > 0).all()


def test_load_runner_warms_every_shape_then_serves_all():
    """run_load serves one small request per shape untimed, forgets it, then
    replays the seeded arrivals; every timed request completes."""
    from cpabdiffeo_b200.serving_load import WARM_BURST, make_requests, run_load
    reqs = make_requests(40.0, 0.3, seed=8, max_points=2e4, reg_steps=12, max_side=96)
    r = run_load(reqs, device=torch.device(DEV), time_limit_s=60.0)
    shapes = {(q.dim, tuple(q.nCs), q.tess) for _, q in reqs if isinstance(q, TransformRequest)}
    has_reg = any(isinstance(q, RegistrationRequest) for _, q in reqs)
    max_jobs = inspect.signature(CpabServer.__init__).parameters["max_jobs"].default
    assert r["warm_up_requests"] == len(shapes) + max_jobs * int(has_reg) + WARM_BURST
    assert r["requests_done"] == r["requests_submitted"] == len(reqs)


def test_inflight_point_bound_admits_in_order_and_drains():
    """Transforms are admitted in arrival order while at most
    max_inflight_points are in flight; a registration queued behind held-back
    transforms still starts; everything drains and the count returns to 0."""
    rng = np.random.default_rng(3)
    geo = build_space(1, (100,), "II")
    theta = Prior.create(geo, 0.1, 1.0).sample(12, rng)
    srv = CpabServer(device=DEV, max_inflight_points=20_000)
    ids = [srv.submit(TransformRequest(1, (100,), theta[i], rng.uniform(0, 1, (8000, 1)).astype(np.float32)))
           for i in range(12)]
    src = gaussian_filter(rng.uniform(0, 1, (32, 32)).astype(np.float32), 3.0)
    jid = srv.submit(RegistrationRequest(src, np.roll(src, 1, axis=1), n_steps=4, seed=5))
    srv.step()
    assert srv.tr_points == 16_000 and len(srv.waiting) == 10      # two transforms fit, ten wait
    assert all(r.rid != jid for r in srv.waiting)                  # the job was not held back
    peak = 0
    while not srv.idle():
        srv.step()
        peak = max(peak, srv.tr_points)
    assert len(srv.done) == 13 and srv.tr_points == 0 and srv.in_use == 0
    assert peak <= 20_000
    t_admit = [srv.done[i].t_admit for i in ids]
    assert all(a <= b for a, b in zip(t_admit, t_admit[1:]))
    assert set(srv.host_seconds) == {"retire", "admit", "launch", "jobs"}
