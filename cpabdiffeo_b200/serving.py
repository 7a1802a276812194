"""Continuous-batching request loop for CPAB transforms and registrations.

Requests of mixed dimension, tessellation and size arrive at any time
(`submit`).  Each scheduler iteration (`step`):
  1. retires finished work (CUDA events) and frees its device-memory share;
  2. admits waiting requests in arrival order while their estimated device
     memory fits the budget and, for transforms, while the points admitted
     and not yet finished stay under max_inflight_points -- work that arrives
     while other work is on the GPU joins as soon as room frees up, and one
     iteration never packs more than that many points on the host (under
     overload the excess waits in the queue instead of stalling the loop);
  3. launches all admitted transform requests that share a space (dim, cells,
     tessellation, precision, sign, integration parameters) as ONE ragged
     batch (one prologue launch for all thetas, one persistent integration
     launch) on a free lane -- a high-priority stream with its own pinned and
     device buffers, reused batch after batch, so launches allocate nothing;
  4. advances every running registration job by a slice of MCMC steps on a
     low-priority stream, one slice in flight per job, so registration slices
     and transform batches overlap and transform batches (high-priority
     streams) are not queued behind long registrations: priority orders
     kernels, and the registration kernels run capped at a share of the SMs
     (the rest stays free for transform batches); at most max_jobs jobs run
     at once, further ones wait without blocking the transforms behind them.
No call of the loop waits for the device: inputs go through pinned host
buffers with asynchronous copies (a copy from pageable memory would wait for
the whole stream, and so stall every request behind a registration slice),
completion is polled with events.
State kept resident on the GPU: the basis of each space, every job's theta,
log-likelihood and chain state, each registration space's proposal scales.
Results do not depend on what else was in the batch: the transform kernels
are per point, the likelihood reduction has a fixed order per image, and
each job's random stream is keyed by its own seed (tests/test_gpu_serving.py
checks alone == in the mix).
"""
from __future__ import annotations

import itertools
import os
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .cpa_space import CpaSpace
from .mcmc import BatchedMetropolis
from .registration import GaussianLogLikelihood
from .space import Prior


@dataclass
class TransformRequest:
    dim: int
    nCs: tuple
    theta: np.ndarray                  # [d]
    pts: np.ndarray                    # [n, dim] float32 or float64
    tess: str = "II"
    sign: int = 1
    scheme: str = "auto"               # auto: closed form in 1D, the reference's calc_T scheme otherwise
    params: dict = field(default_factory=lambda: dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100))


@dataclass
class RegistrationRequest:
    src: np.ndarray                    # [H, W] float32
    dst: np.ndarray                    # [H, W] float32
    n_steps: int = 200
    sigma: float = 0.05
    scale: float = 0.05
    seed: int = 0
    nCs: tuple = (4, 4)
    tess: str = "I"
    rule: str = "reference"
    params: dict = field(default_factory=lambda: dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100))


@dataclass
class _Record:
    rid: int
    req: object
    t_submit: float
    bytes: int
    points: int = 0                    # transform points (0 for registrations)
    t_admit: float = 0.0
    t_done: float = 0.0
    result: object = None


class _Lane:
    """One transform stream and the buffers a batch on it uses: pinned and
    device points in and out, thetas, offsets, tables and workspace.  A lane
    runs one batch at a time and the next batch reuses its buffers once the
    previous one has retired, so launching allocates nothing once the
    buffers have reached the sizes the traffic needs (they grow to powers of
    two; reserve() and the warm-up size them ahead of traffic)."""

    def __init__(self, device, stream):
        self.device, self.stream = device, stream
        self.busy = False
        self.bufs: dict = {}

    def buf(self, name: str, numel: int, dtype, pinned: bool = False) -> torch.Tensor:
        key = (name, dtype)
        b = self.bufs.get(key)
        if b is None or b.numel() < numel:
            n = 1 << max(12, (max(numel, 1) - 1).bit_length())
            if pinned:
                b = torch.empty(n, dtype=dtype).pin_memory()
            else:
                with torch.cuda.stream(self.stream):
                    b = torch.empty(n, dtype=dtype, device=self.device)
            self.bufs[key] = b
        return b


class CpabServer:
    """max_jobs: registration jobs running at once (more wait, in arrival
    order, while transforms keep being admitted); job_sm_fraction: the share
    of the SMs one registration slice's kernels may occupy (their launches --
    captured in CUDA graphs -- are capped at that many CTAs), so transform
    batches on the high-priority streams find free SMs instead of waiting for
    a registration kernel to drain.  max_inflight_points: transform points
    admitted and not yet finished (the device-side queue depth; more wait on
    the host, in arrival order).  The defaults (4 jobs of at most 15 % of the
    SMs each) leave 40 % of the SMs to transforms at all times: measured on
    the mix at 200 req/s, transform p99 39 ms against 200 ms with 8 jobs of
    25 % (which can occupy every SM), at the price of slower registrations;
    batches and the in-flight depth of 2^21 points bound the host work of one
    iteration (measured transform p99 17-21 ms against 40-300 ms at 2^22;
    with the lanes and reserve() below, 9.5-12 ms).  max_batch_requests:
    requests per batch (the lanes' per-request buffers are sized for it).
    copy_threads: host threads that pack inputs into and unpack results out
    of the pinned buffers (numpy copies release the GIL); 0: min(8, cores)."""

    def __init__(self, device=None, memory_budget_bytes: int | None = None, n_streams: int = 4,
                 mcmc_slice: int = 20, max_batch_points: int = 1 << 21, max_jobs: int = 4,
                 job_sm_fraction: float = 0.15, max_inflight_points: int = 1 << 21, copy_threads: int = 0,
                 max_batch_requests: int = 64):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if memory_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            memory_budget_bytes = int(free * 0.5)
        self.budget = int(memory_budget_bytes)
        self.in_use = 0
        # transforms: high-priority streams; registration slices: low priority
        self.streams = [torch.cuda.Stream(device=self.device, priority=-1) for _ in range(n_streams)]
        self.job_streams = [torch.cuda.Stream(device=self.device, priority=0) for _ in range(n_streams)]
        # job images are staged (pinned fill, copy in on a stream of their own,
        # which the job's stream then waits for) by a worker thread: that copy
        # call has been seen to block the host for tens of ms under load
        self._job_copy_stream = torch.cuda.Stream(device=self.device, priority=0)
        self._stage_pool = ThreadPoolExecutor(max_workers=1)
        self._rr_jobs = itertools.cycle(range(n_streams))
        self._pinned: dict = {}
        self.lanes = [_Lane(self.device, st) for st in self.streams]
        self._lane_next = 0
        self.max_batch_requests = int(max_batch_requests)
        self._job_slots: list = []         # free (src, dst) device image buffers for registration jobs
        self.mcmc_slice = int(mcmc_slice)
        self.max_batch_points = int(max_batch_points)
        self._ids = itertools.count()
        self.waiting: deque[_Record] = deque()
        self.ready_transforms: list[_Record] = []
        self.inflight: list[tuple[torch.cuda.Event, list, object]] = []
        self.jobs: list[dict] = []
        self.done: dict[int, _Record] = {}
        self._spaces: dict = {}
        self._priors: dict = {}
        self.max_jobs = int(max_jobs)
        self._finishing = 0                # jobs whose last slice is enqueued, not yet retired
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.job_max_ctas = max(1, int(sms * job_sm_fraction))
        self.max_inflight_points = int(max_inflight_points)
        self.tr_points = 0                 # transform points admitted and not yet retired
        self._prop_std: dict = {}
        # host seconds spent in each phase of step(), in total and in the longest
        # single call (the loop polls, so totals follow the wall time; a long
        # single call -- packing a large batch, starting a job -- holds back
        # every request behind it)
        self.host_seconds = dict(retire=0.0, admit=0.0, launch=0.0, jobs=0.0)
        self.host_max_seconds = dict(retire=0.0, admit=0.0, launch=0.0, jobs=0.0, pack=0.0, enqueue=0.0,
                                     unpack=0.0, job_start=0.0, job_slice=0.0, job_pin=0.0, job_ll=0.0,
                                     job_chain=0.0)
        n_copy = int(copy_threads) if copy_threads > 0 else min(8, os.cpu_count() or 1)
        self._copy_pool = ThreadPoolExecutor(max_workers=n_copy) if n_copy > 1 else None

    # ---------------------------------------------------------------- helpers
    def space(self, dim, nCs, tess, precision, for_jobs: bool = False) -> CpaSpace:
        """The space of a request shape; registration jobs get their own
        context, whose persistent launches are capped at job_max_ctas CTAs."""
        key = (dim, tuple(nCs), tess, precision, for_jobs)
        sp = self._spaces.get(key)
        if sp is None:
            sp = CpaSpace([0.0] * dim, [1.0] * dim, tuple(nCs), tess=tess, device=self.device, precision=precision)
            if for_jobs:
                sp.set_launch(max_ctas=self.job_max_ctas)
            self._spaces[key] = sp
        return sp

    def prior(self, sp: CpaSpace) -> Prior:
        key = sp.geo.subspace_string
        if key not in self._priors:
            self._priors[key] = Prior.create(sp.geo, 0.1, 1.0)
        return self._priors[key]

    def _pinned_buf(self, numel: int, dtype) -> torch.Tensor:
        """A pinned host buffer of at least numel elements from a reusable pool
        (sizes are powers of two, so released buffers fit later requests)."""
        free = self._pinned.setdefault(dtype, [])
        best = None
        for i, b in enumerate(free):
            if b.numel() >= numel and (best is None or b.numel() < free[best].numel()):
                best = i
        if best is not None:
            return free.pop(best)
        return torch.empty(1 << max(16, (max(numel, 1) - 1).bit_length()), dtype=dtype).pin_memory()

    def reserve(self, dims: int = 3, image_side: int = 0, dtypes=(torch.float32,),
                largest_request_values: int = 0) -> None:
        """Allocates ahead of traffic what a loaded server otherwise allocates
        while requests wait (pinned allocations can take tens of ms): every
        lane's pinned and device point buffers for a full batch of `dims`-D
        points (or the largest single request, points x dim values, when that
        is larger: a request above max_batch_points is a batch of its own),
        pinned staging for max_jobs image pairs of side image_side, and device
        images for them."""
        n = max(self.max_batch_points * dims, int(largest_request_values))
        for dt in dtypes:
            for lane in self.lanes:
                for name in ("pin_x", "pin_o"):
                    lane.buf(name, n, dt, pinned=True)
                for name in ("dev_x", "dev_o"):
                    lane.buf(name, n, dt)
        if image_side > 0:
            n_img = image_side * image_side
            self._release_pinned(*[self._pinned_buf(n_img, torch.float32) for _ in range(2 * self.max_jobs)])
            while len(self._job_slots) < self.max_jobs:
                self._job_slots.append((torch.empty(n_img, dtype=torch.float32, device=self.device),
                                        torch.empty(n_img, dtype=torch.float32, device=self.device)))
        # job results (theta, ll, accepted count)
        self._release_pinned(*[self._pinned_buf(1, torch.float64) for _ in range(2 * self.max_jobs)],
                             *[self._pinned_buf(1, torch.int64) for _ in range(self.max_jobs)])

    def spread_lane_buffers(self) -> None:
        """Grows every lane's buffers to the largest size any lane holds for
        the same buffer (after a warm-up, which may have used one lane), and
        the per-request ones (thetas, offsets, tables, workspace) to a batch
        of max_batch_requests requests of the largest transform space served
        so far, so no lane allocates while requests wait."""
        spaces = [sp for (dim, nCs, tess, prec, for_jobs), sp in self._spaces.items() if not for_jobs]
        if spaces:
            m = self.max_batch_requests
            d = max(sp.d for sp in spaces)
            D = max(sp.D for sp in spaces)
            ws = max(int(sp._ctx.lib.cpab_batched_workspace_bytes(m)) for sp in spaces)
            for lane in self.lanes:
                lane.buf("pin_th", m * d, torch.float64, pinned=True)
                lane.buf("pin_off", m + 1, torch.int64, pinned=True)
                lane.buf("dev_th", m * d, torch.float64)
                lane.buf("dev_off", m + 1, torch.int64)
                lane.buf("dev_sA", m * D, torch.float64)
                lane.buf("dev_Tr", m * D, torch.float64)
                lane.buf("dev_ws", ws, torch.uint8)
        sizes: dict = {}
        for lane in self.lanes:
            for key, b in lane.bufs.items():
                sizes[key] = max(sizes.get(key, 0), b.numel())
        for lane in self.lanes:
            for (name, dt), n in sizes.items():
                lane.buf(name, n, dt, pinned=name.startswith("pin_"))

    def _note(self, key: str, t0: float) -> None:
        d = time.perf_counter() - t0
        if d > self.host_max_seconds[key]:
            self.host_max_seconds[key] = d

    def _copy_many(self, pairs) -> None:
        """dst[...] = src for every (dst, src) pair (same shape; dtype cast as
        needed); large pairs are cut in row chunks of about 2^20 elements
        that the copy threads run in parallel, small ones are copied here."""
        chunks = []
        for dst, src in pairs:
            row = max(1, dst[0].size) if dst.ndim > 1 and dst.shape[0] else 1
            n = dst.shape[0]
            if self._copy_pool is None or n * row < (1 << 18):
                np.copyto(dst, src, casting="unsafe")
                continue
            step = max(1, (1 << 20) // row)
            chunks.extend((dst[a:a + step], src[a:a + step]) for a in range(0, n, step))
        if chunks:
            list(self._copy_pool.map(lambda c: np.copyto(c[0], c[1], casting="unsafe"), chunks))

    def close(self) -> None:
        """Stops the copy threads (the server is not used afterwards)."""
        if self._copy_pool is not None:
            self._copy_pool.shutdown(wait=True)
            self._copy_pool = None
        if self._stage_pool is not None:
            self._stage_pool.shutdown(wait=True)
            self._stage_pool = None

    def _release_pinned(self, *bufs) -> None:
        for b in bufs:
            self._pinned.setdefault(b.dtype, []).append(b)

    @staticmethod
    def _estimate_bytes(req) -> int:
        if isinstance(req, TransformRequest):
            n = int(np.asarray(req.pts).shape[0])
            return 2 * n * req.dim * np.asarray(req.pts).dtype.itemsize + (1 << 16)
        H, W = np.shape(req.src)
        return 4 * H * W * 4 + (1 << 20)

    # ---------------------------------------------------------------- API
    def submit(self, req, t_submit: float | None = None) -> int:
        rid = next(self._ids)
        n = int(np.asarray(req.pts).shape[0]) if isinstance(req, TransformRequest) else 0
        self.waiting.append(_Record(rid, req, time.perf_counter() if t_submit is None else t_submit,
                                    self._estimate_bytes(req), n))
        return rid

    def idle(self) -> bool:
        return not (self.waiting or self.ready_transforms or self.inflight or self.jobs)

    def step(self) -> None:
        hs = self.host_seconds
        t0 = time.perf_counter()
        self._retire()
        t1 = time.perf_counter()
        self._admit()
        t2 = time.perf_counter()
        self._launch_transforms()
        t3 = time.perf_counter()
        self._advance_jobs()
        t4 = time.perf_counter()
        hm = self.host_max_seconds
        for k, d in (("retire", t1 - t0), ("admit", t2 - t1), ("launch", t3 - t2), ("jobs", t4 - t3)):
            hs[k] += d
            if d > hm[k]:
                hm[k] = d

    def run_until_idle(self, timeout_s: float = 600.0) -> None:
        t0 = time.perf_counter()
        while not self.idle():
            self.step()
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError("server did not drain")

    def latencies(self) -> np.ndarray:
        return np.asarray([r.t_done - r.t_submit for r in self.done.values()])

    # ---------------------------------------------------------------- scheduler
    def _retire(self) -> None:
        still = []
        for ev, recs, finalize in self.inflight:
            if ev.query():
                finalize()
                now = time.perf_counter()
                for r in recs:
                    r.t_done = now
                    self.done[r.rid] = r
                    self.in_use -= r.bytes
                    self.tr_points -= r.points
            else:
                still.append((ev, recs, finalize))
        self.inflight = still

    def _admit(self) -> None:
        """Admit waiting requests in arrival order while their memory fits;
        a registration finding max_jobs jobs running stays queued (in order)
        without holding back the transforms behind it, and transforms stop
        being admitted (in order) once max_inflight_points are in flight,
        without holding back the registrations behind them."""
        kept: deque[_Record] = deque()
        # finishing jobs (last slice enqueued, not retired) still hold their
        # image slot and pinned buffers, so they count
        jobs = len(self.jobs) + self._finishing
        tr_full = False
        started = False                    # one job start per iteration: the loop turns between starts
        while self.waiting:
            r = self.waiting.popleft()
            is_job = not isinstance(r.req, TransformRequest)
            if is_job and (jobs >= self.max_jobs or started):
                kept.append(r)
                continue
            if not is_job and (tr_full or (self.tr_points > 0 and
                                           self.tr_points + r.points > self.max_inflight_points)):
                tr_full = True
                kept.append(r)
                continue
            if self.in_use + r.bytes > self.budget and self.in_use > 0:
                kept.append(r)             # wait for memory to free up (always admit when idle)
                kept.extend(self.waiting)
                self.waiting.clear()
                break
            r.t_admit = time.perf_counter()
            self.in_use += r.bytes
            self.tr_points += r.points
            if is_job:
                t_js = time.perf_counter()
                self._start_job(r)
                self._note("job_start", t_js)
                jobs += 1
                started = True
            else:
                self.ready_transforms.append(r)
        self.waiting = kept

    def _launch_transforms(self) -> None:
        """Groups the admitted transforms by space into batches (at most
        max_batch_points points and max_batch_requests requests) and launches
        each on a free lane; batches without a free lane wait (admitted, in
        order) for the next iteration."""
        if not self.ready_transforms:
            return
        groups: dict = {}
        for r in self.ready_transforms:
            q: TransformRequest = r.req
            prec = torch.float64 if np.asarray(q.pts).dtype == np.float64 else torch.float32
            scheme = q.scheme
            if scheme == "auto":
                scheme = "exact" if q.dim == 1 else "ref"
            key = (q.dim, tuple(q.nCs), q.tess, prec, int(q.sign), scheme, tuple(sorted(q.params.items())))
            groups.setdefault(key, []).append(r)
        waiting = []
        for key, recs in groups.items():
            batches, batch, npts = [], [], 0
            for r in recs:
                if batch and (npts + r.points > self.max_batch_points or len(batch) >= self.max_batch_requests):
                    batches.append(batch)
                    batch, npts = [], 0
                batch.append(r)
                npts += r.points
            if batch:
                batches.append(batch)
            for b in batches:
                # lanes in rotation (the first free one from a rotating start), so every lane stays warm
                lane = next((ln for ln in self._lane_order() if not ln.busy), None)
                if lane is None:
                    waiting.extend(b)
                else:
                    self._launch_group(lane, key, b)
        self.ready_transforms = waiting

    def _lane_order(self):
        k = self._lane_next
        self._lane_next = (k + 1) % len(self.lanes)
        return self.lanes[k:] + self.lanes[:k]

    def _launch_group(self, lane: _Lane, key, recs) -> None:
        dim, nCs, tess, prec, sign, scheme, params = key
        params = dict(params)
        sp = self.space(dim, nCs, tess, prec)
        np_dt = np.float64 if prec == torch.float64 else np.float32
        n = len(recs)
        offs = np.concatenate([[0], np.cumsum([r.points for r in recs])]).astype(np.int64)
        total = int(offs[-1])
        tdt = prec
        lane.busy = True
        t_pack = time.perf_counter()
        pin_x = lane.buf("pin_x", total * dim, tdt, pinned=True)
        pin_o = lane.buf("pin_o", total * dim, tdt, pinned=True)
        pin_th = lane.buf("pin_th", n * sp.d, torch.float64, pinned=True)
        pin_off = lane.buf("pin_off", n + 1, torch.int64, pinned=True)
        xv = pin_x[:total * dim].numpy().reshape(total, dim)
        self._copy_many([(xv[a:b], np.asarray(r.req.pts).reshape(-1, dim))
                         for r, a, b in zip(recs, offs[:-1], offs[1:])])
        pin_th[:n * sp.d].numpy().reshape(n, sp.d)[:] = np.stack([np.asarray(r.req.theta, dtype=np.float64)
                                                                  for r in recs])
        pin_off[:n + 1].numpy()[:] = offs
        self._note("pack", t_pack)
        t_enq = time.perf_counter()
        ws_bytes = int(sp._ctx.lib.cpab_batched_workspace_bytes(n))
        dx = lane.buf("dev_x", total * dim, tdt)
        do = lane.buf("dev_o", total * dim, tdt)
        dth = lane.buf("dev_th", n * sp.d, torch.float64)
        doff = lane.buf("dev_off", n + 1, torch.int64)
        dsA = lane.buf("dev_sA", n * sp.D, torch.float64)
        dTr = lane.buf("dev_Tr", n * sp.D, torch.float64)
        ws = lane.buf("dev_ws", ws_bytes, torch.uint8)
        sch = {"exact": _lib.SCHEME_EXACT, "ref": _lib.SCHEME_REF, "simple": _lib.SCHEME_SIMPLE}[scheme]
        with torch.cuda.stream(lane.stream):
            x = dx[:total * dim].view(total, dim)
            x.copy_(pin_x[:total * dim].view(total, dim), non_blocking=True)
            th = dth[:n * sp.d].view(n, sp.d)
            th.copy_(pin_th[:n * sp.d].view(n, sp.d), non_blocking=True)
            off = doff[:n + 1]
            off.copy_(pin_off[:n + 1], non_blocking=True)
            out = do[:total * dim].view(total, dim)
            tables = sp.tables_from_theta(th, float(params["dt"]), sign,
                                          out=(dsA[:n * sp.D].view(n, sp.D), dTr[:n * sp.D].view(n, sp.D)))
            sp.calc_T_batched(tables, x, out, offsets=off, workspace=ws, scheme=sch, **params)
            pin_o[:total * dim].view(total, dim).copy_(out, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(lane.stream)
        self._note("enqueue", t_enq)

        def finalize(recs=recs, offs=offs, pin_o=pin_o, total=total, lane=lane):
            t_un = time.perf_counter()
            res = pin_o[:total * dim].numpy().reshape(total, dim)
            for r, a, b in zip(recs, offs[:-1], offs[1:]):
                r.result = np.empty((b - a, dim), dtype=np_dt)
            self._copy_many([(r.result, res[a:b]) for r, a, b in zip(recs, offs[:-1], offs[1:])])
            lane.busy = False                  # its buffers may be reused from here on
            self._note("unpack", t_un)
        self.inflight.append((ev, recs, finalize))

    def _start_job(self, r: _Record) -> None:
        """Starts a registration job: its image pair is staged into a reserved
        device slot by the staging thread (the job waits in state "staging"),
        or, without a free slot, copied in on the job's stream here."""
        q: RegistrationRequest = r.req
        sp = self.space(2, q.nCs, q.tess, torch.float32, for_jobs=True)
        stream = self.job_streams[next(self._rr_jobs)]
        key = sp.geo.subspace_string
        if key not in self._prop_std:
            # once per space, outside any job stream's work
            self._prop_std[key] = torch.as_tensor(np.sqrt(np.diag(self.prior(sp).cov_cpa)), device=self.device)
        src_h, dst_h = np.asarray(q.src, dtype=np.float32), np.asarray(q.dst, dtype=np.float32)
        H, W = src_h.shape
        t0 = time.perf_counter()
        pins = (self._pinned_buf(H * W, torch.float32), self._pinned_buf(H * W, torch.float32))
        self._note("job_pin", t0)
        # a reserved device image slot when one fits (released when the job
        # retires, after its last kernel), else fresh device memory
        i_slot = next((i for i, sl in enumerate(self._job_slots) if sl[0].numel() >= H * W), None)
        slot = self._job_slots.pop(i_slot) if i_slot is not None else None
        job = dict(rec=r, sp=sp, stream=stream, left=int(q.n_steps), ev=None, pins=pins, slot=slot, mh=None)
        if slot is not None:
            src, dst = slot[0][:H * W].view(H, W), slot[1][:H * W].view(H, W)
            staged = torch.cuda.Event()

            def stage(src=src, dst=dst, staged=staged):
                pins[0][:H * W].numpy()[:] = src_h.ravel()
                pins[1][:H * W].numpy()[:] = dst_h.ravel()
                with torch.cuda.device(self.device), torch.cuda.stream(self._job_copy_stream):
                    src.copy_(pins[0][:H * W].view(H, W), non_blocking=True)
                    dst.copy_(pins[1][:H * W].view(H, W), non_blocking=True)
                    staged.record(self._job_copy_stream)
            job.update(keep=(src, dst), staged=staged, staging=self._stage_pool.submit(stage))
        else:
            pins[0][:H * W].numpy()[:] = src_h.ravel()
            pins[1][:H * W].numpy()[:] = dst_h.ravel()
            with torch.cuda.stream(stream):
                src = pins[0][:H * W].view(H, W).to(self.device, non_blocking=True)
                dst = pins[1][:H * W].view(H, W).to(self.device, non_blocking=True)
            job.update(keep=(src, dst), staged=None, staging=None)
        self.jobs.append(job)

    def _build_chain(self, job) -> None:
        """The job's likelihood and chain on its stream, once its images are in."""
        q: RegistrationRequest = job["rec"].req
        sp, stream = job["sp"], job["stream"]
        if job["staged"] is not None:
            job["staging"].result()                # re-raises a staging error
            stream.wait_event(job["staged"])
        src, dst = job["keep"]
        with torch.cuda.stream(stream):
            t1 = time.perf_counter()
            ll = GaussianLogLikelihood(sp, src, dst, q.sigma, params_flow_int=q.params)
            self._note("job_ll", t1)
            t2 = time.perf_counter()
            job["mh"] = BatchedMetropolis(ll, torch.zeros((1, sp.d), dtype=torch.float64, device=self.device),
                                          self._prop_std[sp.geo.subspace_string], scale=q.scale, seed=q.seed,
                                          rule=q.rule)
            self._note("job_chain", t2)

    def _advance_jobs(self) -> None:
        running = []
        for job in self.jobs:
            if job["mh"] is None:
                if job["staging"] is not None and not job["staging"].done():
                    running.append(job)        # images still being staged
                    continue
                self._build_chain(job)
            if job["ev"] is not None and not job["ev"].query():
                running.append(job)            # one slice in flight per job
                continue
            k = min(self.mcmc_slice, job["left"])
            with torch.cuda.stream(job["stream"]):
                mh = job["mh"]
                t_sl = time.perf_counter()
                if k == self.mcmc_slice and job.get("warm"):
                    # full slices replay a CUDA graph captured on this stream (one host call per slice)
                    if mh._graph is None:
                        mh.capture(self.mcmc_slice)
                    mh._graph.replay()
                else:
                    mh.run(k)
                    job["warm"] = True
                self._note("job_slice", t_sl)
                job["left"] -= k
                if job["left"] == 0:
                    self._finishing += 1
                    mh = job["mh"]
                    d = mh.theta.numel()
                    th_h = self._pinned_buf(d, torch.float64)
                    ll_h = self._pinned_buf(1, torch.float64)
                    acc_h = self._pinned_buf(1, torch.int64)
                    th_h[:d].copy_(mh.theta.reshape(-1), non_blocking=True)
                    ll_h[:1].copy_(mh.ll.reshape(-1)[:1], non_blocking=True)
                    acc_h[:1].copy_(mh.n_accepted.reshape(-1)[:1], non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(job["stream"])

                    def finalize(rec=job["rec"], th_h=th_h, ll_h=ll_h, acc_h=acc_h, d=d, keep=(mh, job["keep"]),
                                 pins=job["pins"], slot=job["slot"]):
                        rec.result = dict(theta=th_h[:d].numpy().copy(), ll=float(ll_h[0]),
                                          accepted=int(acc_h[0]))
                        self._release_pinned(th_h, ll_h, acc_h, *pins)
                        self._finishing -= 1
                        if slot is not None:
                            self._job_slots.append(slot)
                    self.inflight.append((ev, [job["rec"]], finalize))
                else:
                    job["ev"] = torch.cuda.Event()
                    job["ev"].record(job["stream"])
                    running.append(job)
        self.jobs = running
