"""Seeded open-loop load for the continuous-batching server: Poisson arrivals
of a mixed request stream, replayed in real time; reports latency
percentiles and throughput.

Mix (the serving configuration): each request is 1D, 2D or 3D with equal
probability and nC drawn from {16, 64, 256, 1024}, mapped to grids
  1D: nC cells;  2D tess I: 2x2, 4x4, 8x8, 16x16 boxes (4 triangles each);
  3D tess II: (4,2,2), (4,4,4), (8,8,4) and (8,8,8) boxes -- type II because
  5 tetrahedra per box cannot make these counts; the largest uses 512 cells
  instead of 1024 to keep the dense null-space construction of its basis
  under a minute.
Payload log-uniform in [1e3, 4e6] points (FP32); 10% of the requests are
registration jobs (a float32 image pair, side uniform in [64, 1024], 200
Metropolis steps); theta from the Gaussian prior.
"""
from __future__ import annotations

import gc
import time

import numpy as np
import torch
from scipy.ndimage import gaussian_filter

from .serving import CpabServer, RegistrationRequest, TransformRequest
from .space import Prior, build_space

GRIDS = {
    1: [((16,), "II"), ((64,), "II"), ((256,), "II"), ((1024,), "II")],
    2: [((2, 2), "I"), ((4, 4), "I"), ((8, 8), "I"), ((16, 16), "I")],
    3: [((4, 2, 2), "II"), ((4, 4, 4), "II"), ((8, 8, 4), "II"), ((8, 8, 8), "II")],
}


def make_requests(rate_hz: float, duration_s: float, seed: int = 4, max_points: float = 4e6,
                  reg_fraction: float = 0.1, reg_steps: int = 200, max_side: int = 1024):
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    priors = {}
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t > duration_s:
            break
        if rng.uniform() < reg_fraction:
            side = int(rng.integers(64, max_side + 1))
            src = gaussian_filter(rng.uniform(0, 1, (side, side)).astype(np.float32), 8.0)
            dst = np.roll(src, 2, axis=1) + rng.normal(0, 0.02, (side, side)).astype(np.float32)
            out.append((t, RegistrationRequest(src, dst, n_steps=reg_steps, seed=int(rng.integers(1 << 31)))))
            continue
        dim = int(rng.integers(1, 4))
        nCs, tess = GRIDS[dim][int(rng.integers(0, 4))]
        key = (dim, nCs, tess)
        if key not in priors:
            priors[key] = Prior.create(build_space(dim, nCs, tess), 0.1, 1.0)
        theta = priors[key].sample(1, rng)[0]
        n = int(10 ** rng.uniform(3, np.log10(max_points)))
        pts = rng.uniform(0, 1, (n, dim)).astype(np.float32)
        out.append((t, TransformRequest(dim, nCs, theta, pts, tess=tess)))
    return out


WARM_BURST = 4


def warm_up(srv: CpabServer, requests) -> int:
    """Serve, untimed, one small request of every transform shape in `requests`,
    a burst of WARM_BURST copies of the largest transform payload, and
    max_jobs short registration jobs on the largest image pair (long enough
    to capture their CUDA graphs), then forget them, after
    CpabServer.reserve for the largest point dimension and image side of
    `requests`: the spaces, the kernels of every variant (loaded on first
    launch), the device and pinned host buffers and the graph path are ready
    before the timed arrivals.  Returns the number of warm-up requests."""
    seen, warm = set(), []
    big = max((r for _, r in requests if isinstance(r, TransformRequest)),
              key=lambda r: np.asarray(r.pts).shape[0], default=None)
    if big is not None:
        warm.extend(TransformRequest(big.dim, big.nCs, big.theta, big.pts, tess=big.tess, scheme=big.scheme)
                    for _ in range(WARM_BURST))
    for _, r in requests:
        if isinstance(r, TransformRequest):
            key = (r.dim, tuple(r.nCs), r.tess, r.scheme)
            if key not in seen:
                seen.add(key)
                warm.append(TransformRequest(r.dim, r.nCs, r.theta, r.pts[:1024], tess=r.tess, scheme=r.scheme))
    regs = [r for _, r in requests if isinstance(r, RegistrationRequest)]
    if regs:
        # one job per job stream, on the largest image pair: every stream's
        # allocations and graph capture happen here
        big_reg = max(regs, key=lambda r: np.size(r.src))
        warm.extend(RegistrationRequest(big_reg.src, big_reg.dst, n_steps=2 * srv.mcmc_slice, seed=1 + j,
                                        nCs=big_reg.nCs, tess=big_reg.tess) for j in range(srv.max_jobs))
    sides = [int(max(np.shape(r.src))) for r in regs]
    trs = [r for _, r in requests if isinstance(r, TransformRequest)]
    srv.reserve(dims=max((r.dim for r in trs), default=1), image_side=max(sides, default=0),
                largest_request_values=max((np.asarray(r.pts).size for r in trs), default=0))
    for q in warm:
        srv.submit(q)
    srv.run_until_idle()
    srv.spread_lane_buffers()
    torch.cuda.synchronize()
    srv.done.clear()
    srv.host_seconds = dict.fromkeys(srv.host_seconds, 0.0)
    srv.host_max_seconds = dict.fromkeys(srv.host_max_seconds, 0.0)
    return len(warm)


def run_load(requests, device=None, time_limit_s: float = 120.0, grace_s: float | None = None,
             server_kwargs: dict | None = None) -> dict:
    """Replay `requests` in real time.  With grace_s None the server drains
    (every request is served); otherwise the run stops grace_s after the
    last arrival and reports what was served by then (an overloaded server
    never drains), with the requests still queued or running.
    server_kwargs: CpabServer's scheduling parameters (max_jobs, ...)."""
    srv = CpabServer(device=device, **(server_kwargs or {}))
    # spaces, kernels and graph capture warmed by one small request of each shape (not timed)
    n_warm = warm_up(srv, requests)
    gc.collect()                                   # garbage of earlier work is not collected inside the window
    # the request stream and the warmed server move out of the cyclic
    # collector's reach (as a latency-sensitive Python server freezes its
    # start-up heap), so a collection inside the window scans only what the
    # window creates; the pauses it still takes are recorded
    gc.freeze()
    pauses = []
    t_gc = [0.0]

    def on_gc(phase, info):
        if phase == "start":
            t_gc[0] = time.perf_counter()
        else:
            pauses.append(time.perf_counter() - t_gc[0])
    gc.callbacks.append(on_gc)
    t0 = time.perf_counter()
    i = 0
    while i < len(requests) or not srv.idle():
        now = time.perf_counter() - t0
        while i < len(requests) and requests[i][0] <= now:
            srv.submit(requests[i][1], t_submit=t0 + requests[i][0])
            i += 1
        srv.step()
        if now > time_limit_s:
            break
        if grace_s is not None and i == len(requests) and now > (requests[-1][0] if requests else 0.0) + grace_s:
            break
    wall = time.perf_counter() - t0
    gc.callbacks.remove(on_gc)
    gc.unfreeze()
    # work still queued or running (an overloaded window) finishes before the
    # server and its device buffers are dropped
    torch.cuda.synchronize(srv.device)
    lat = np.asarray([r.t_done - r.t_submit for r in srv.done.values()])
    pts = sum(int(np.asarray(r.req.pts).shape[0]) for r in srv.done.values() if isinstance(r.req, TransformRequest))
    n_reg = sum(1 for r in srv.done.values() if isinstance(r.req, RegistrationRequest))
    lat_t = np.asarray([r.t_done - r.t_submit for r in srv.done.values() if isinstance(r.req, TransformRequest)])
    srv.close()
    return {
        "requests_submitted": len(requests), "requests_done": len(srv.done), "registrations_done": n_reg,
        "wall_s": wall, "req_per_s": len(srv.done) / wall, "points_per_s": pts / wall,
        "p50_ms": float(np.percentile(lat, 50) * 1e3) if lat.size else None,
        "p99_ms": float(np.percentile(lat, 99) * 1e3) if lat.size else None,
        "transform_p50_ms": float(np.percentile(lat_t, 50) * 1e3) if lat_t.size else None,
        "transform_p99_ms": float(np.percentile(lat_t, 99) * 1e3) if lat_t.size else None,
        "warm_up_requests": n_warm,
        "left_unserved": len(requests) - len(srv.done),
        "left_registrations": sum(1 for _, q in requests if isinstance(q, RegistrationRequest)) - n_reg,
        "host_seconds": {k: round(v, 3) for k, v in srv.host_seconds.items()},
        "host_max_call_ms": {k: round(v * 1e3, 2) for k, v in srv.host_max_seconds.items()},
        "gc_pauses": len(pauses), "gc_max_ms": round(max(pauses, default=0.0) * 1e3, 2),
    }


def capacity_estimate(device=None, reg_sides=(128, 512, 1024), reg_steps: int = 40,
                      server_kwargs: dict | None = None) -> dict:
    """Requests per second one GPU can serve of the mix, from measured service
    times of each request type served alone (host work, copies and kernels,
    one request at a time).

    Transforms: for each (dim, grid) of the mix, the service time of 1e3 and
    1e6 points gives t(n) = o + n / r; the mix's payload is log-uniform in
    [1e3, 4e6] (mean (4e6 - 1e3) / ln 4000).  Registrations: the per-step time
    at a few image sides gives t(side) = a + b side^2; sides are uniform in
    [64, 1024] and each job takes 200 steps plus its start (the per-step time
    is the difference of a 3 x reg_steps and a reg_steps job, so the start --
    staging, first eager slice, graph capture -- is measured apart) -- once
    with the whole GPU and once capped as the server runs them
    (job_sm_fraction of the SMs).
      capacity_req_per_s = 1 / (0.9 E[t_transform] + 0.1 E[t_registration, whole GPU]):
        the device-time bound of the mix, one request at a time;
      capacity_with_job_caps = min(max_jobs / (0.1 E[t_registration, capped]),
                                   (1 - u) / (0.9 E[t_transform])), u = max_jobs * job_sm_fraction:
        the rate the server's scheduling sustains (max_jobs capped jobs at
        once, transforms on the SMs the jobs leave)."""
    kw = dict(server_kwargs or {})
    srv = CpabServer(device=device, **kw)
    whole = CpabServer(device=device, **dict(kw, job_sm_fraction=1.0))
    # buffers sized ahead, as a warmed server has them (the lanes rotate, so
    # repeats land on different lanes)
    for server in (srv, whole):
        server.reserve(dims=3, image_side=max(reg_sides), largest_request_values=3 * 1_000_000)
    rng = np.random.default_rng(11)

    def serve(server, req) -> float:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        server.submit(req)
        server.run_until_idle()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    mean_n = (4e6 - 1e3) / np.log(4000.0)
    per_cfg = {}
    for dim, grids in GRIDS.items():
        for nCs, tess in grids:
            prior = Prior.create(build_space(dim, nCs, tess), 0.1, 1.0)
            theta = prior.sample(1, rng)[0]
            small = rng.uniform(0, 1, (1000, dim)).astype(np.float32)
            big = rng.uniform(0, 1, (1_000_000, dim)).astype(np.float32)
            serve(srv, TransformRequest(dim, nCs, theta, small, tess=tess))     # warm the space and kernels
            srv.spread_lane_buffers()
            ts = min(serve(srv, TransformRequest(dim, nCs, theta, small, tess=tess)) for _ in range(3))
            tb = min(serve(srv, TransformRequest(dim, nCs, theta, big, tess=tess)) for _ in range(2))
            r = (1_000_000 - 1000) / max(tb - ts, 1e-9)
            o = max(ts - 1000 / r, 0.0)
            per_cfg[f"{dim}d_{'x'.join(map(str, nCs))}_{tess}"] = {"overhead_ms": o * 1e3, "points_per_s": r,
                                                                 "mean_ms": (o + mean_n / r) * 1e3}
    t_tr = float(np.mean([v["mean_ms"] for v in per_cfg.values()])) * 1e-3
    e_side2 = (1024 ** 3 - 63 ** 3) / (3 * (1024 - 63))       # E[side^2], side uniform on 64..1024

    def registration(server):
        # per-step time from two job lengths (the difference cancels the job's
        # start: staging, first eager slice, graph capture), plus that start
        per_step, start = {}, {}
        for side in reg_sides:
            src = gaussian_filter(rng.uniform(0, 1, (side, side)).astype(np.float32), 8.0)
            dst = np.roll(src, 2, axis=1)
            serve(server, RegistrationRequest(src, dst, n_steps=2 * server.mcmc_slice, seed=1))  # warm (graph)
            t_short = serve(server, RegistrationRequest(src, dst, n_steps=reg_steps, seed=2))
            t_long = serve(server, RegistrationRequest(src, dst, n_steps=3 * reg_steps, seed=3))
            per_step[side] = max(t_long - t_short, 0.0) / (2 * reg_steps)
            start[side] = max(t_short - reg_steps * per_step[side], 0.0)
        sides = np.array(sorted(per_step))
        b, a = np.polyfit(sides.astype(float) ** 2, [per_step[s] for s in sides], 1)
        t_start = float(np.mean(list(start.values())))
        return (t_start + 200 * (a + b * e_side2), {int(s): v * 1e3 for s, v in per_step.items()},
                t_start * 1e3)

    t_reg, steps_whole, start_whole = registration(whole)
    t_reg_cap, steps_cap, start_cap = registration(srv)
    srv.close()
    whole.close()
    mean_t = 0.9 * t_tr + 0.1 * t_reg
    sms = torch.cuda.get_device_properties(srv.device).multi_processor_count
    u = min(1.0, srv.max_jobs * srv.job_max_ctas / sms)
    r_reg = srv.max_jobs / (0.1 * t_reg_cap)
    r_tr = (1.0 - u) / (0.9 * t_tr) if u < 1.0 else float("inf")
    return {"transform_mean_ms": t_tr * 1e3, "registration_mean_ms": t_reg * 1e3,
            "registration_mean_ms_capped": t_reg_cap * 1e3,
            "registration_step_ms": steps_whole, "registration_step_ms_capped": steps_cap,
            "registration_start_ms": start_whole, "registration_start_ms_capped": start_cap,
            "mean_service_ms": mean_t * 1e3, "capacity_req_per_s": 1.0 / mean_t,
            "capacity_with_job_caps": min(r_reg, r_tr),
            "job_caps": {"max_jobs": srv.max_jobs, "ctas_per_job": srv.job_max_ctas, "sm_share_of_jobs": u},
            "device_seconds_per_second_at_2000_req_per_s": 2000 * mean_t,
            "transforms": per_cfg}
