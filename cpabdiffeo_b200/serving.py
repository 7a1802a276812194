"""Continuous-batching request loop for CPAB transforms and registrations.

Requests of mixed dimension, tessellation and size arrive at any time
(`submit`).  Each scheduler iteration (`step`):
  1. retires finished work (CUDA events) and frees its device-memory share;
  2. admits waiting requests in arrival order while their estimated device
     memory fits the budget -- work that arrives while other work is on the
     GPU joins as soon as memory frees up;
  3. launches all admitted transform requests that share a space (dim, cells,
     tessellation, precision, sign, integration parameters) as ONE ragged
     batch (one prologue launch for all thetas, one persistent integration
     launch), on a stream of a small pool, with pinned-memory copies;
  4. advances every running registration job by a slice of MCMC steps on a
     low-priority stream, one slice in flight per job, so registration slices
     and transform batches overlap and transform batches (high-priority
     streams) are not queued behind long registrations: priority orders
     kernels, and the registration kernels run capped at a share of the SMs
     (the rest stays free for transform batches); at most max_jobs jobs run
     at once, further ones wait without blocking the transforms behind them.
State kept resident on the GPU: the basis of each space, every job's theta,
log-likelihood and chain state.  Results do not depend on what else was in
the batch: the transform kernels are per point, the likelihood reduction has
a fixed order per image, and each job's random stream is keyed by its own
seed (tests/test_gpu_serving.py checks alone == in the mix).
"""
from __future__ import annotations

import itertools
import time
from collections import deque
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
    t_admit: float = 0.0
    t_done: float = 0.0
    result: object = None


class CpabServer:
    """max_jobs: registration jobs running at once (more wait, in arrival
    order, while transforms keep being admitted); job_sm_fraction: the share
    of the SMs one registration slice's kernels may occupy (their launches --
    captured in CUDA graphs -- are capped at that many CTAs), so transform
    batches on the high-priority streams find free SMs instead of waiting for
    a registration kernel to drain."""

    def __init__(self, device=None, memory_budget_bytes: int | None = None, n_streams: int = 4,
                 mcmc_slice: int = 20, max_batch_points: int = 1 << 26, max_jobs: int = 8,
                 job_sm_fraction: float = 0.25):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if memory_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            memory_budget_bytes = int(free * 0.5)
        self.budget = int(memory_budget_bytes)
        self.in_use = 0
        # transforms: high-priority streams; registration slices: low priority
        self.streams = [torch.cuda.Stream(device=self.device, priority=-1) for _ in range(n_streams)]
        self.job_streams = [torch.cuda.Stream(device=self.device, priority=0) for _ in range(n_streams)]
        self._rr = itertools.cycle(range(n_streams))
        self._rr_jobs = itertools.cycle(range(n_streams))
        self._pinned: dict = {}
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
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.job_max_ctas = max(1, int(sms * job_sm_fraction))

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
        """A pinned host buffer of at least numel elements from a reusable pool."""
        free = self._pinned.setdefault(dtype, [])
        for i, b in enumerate(free):
            if b.numel() >= numel:
                return free.pop(i)
        return torch.empty(max(numel, 1 << 16), dtype=dtype).pin_memory()

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
        self.waiting.append(_Record(rid, req, time.perf_counter() if t_submit is None else t_submit,
                                    self._estimate_bytes(req)))
        return rid

    def idle(self) -> bool:
        return not (self.waiting or self.ready_transforms or self.inflight or self.jobs)

    def step(self) -> None:
        self._retire()
        self._admit()
        self._launch_transforms()
        self._advance_jobs()

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
            else:
                still.append((ev, recs, finalize))
        self.inflight = still

    def _admit(self) -> None:
        """Admit waiting requests in arrival order while their memory fits;
        a registration finding max_jobs jobs running stays queued (in order)
        without holding back the transforms behind it."""
        kept: deque[_Record] = deque()
        jobs = len(self.jobs)
        while self.waiting:
            r = self.waiting.popleft()
            is_job = not isinstance(r.req, TransformRequest)
            if is_job and jobs >= self.max_jobs:
                kept.append(r)
                continue
            if self.in_use + r.bytes > self.budget and self.in_use > 0:
                kept.append(r)             # wait for memory to free up (always admit when idle)
                kept.extend(self.waiting)
                self.waiting.clear()
                break
            r.t_admit = time.perf_counter()
            self.in_use += r.bytes
            if is_job:
                self._start_job(r)
                jobs += 1
            else:
                self.ready_transforms.append(r)
        self.waiting = kept

    def _launch_transforms(self) -> None:
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
        self.ready_transforms = []
        for key, recs in groups.items():
            # split very large groups
            batch, npts = [], 0
            for r in recs:
                n = int(np.asarray(r.req.pts).shape[0])
                if batch and npts + n > self.max_batch_points:
                    self._launch_group(key, batch)
                    batch, npts = [], 0
                batch.append(r)
                npts += n
            if batch:
                self._launch_group(key, batch)

    def _launch_group(self, key, recs) -> None:
        dim, nCs, tess, prec, sign, scheme, params = key
        params = dict(params)
        sp = self.space(dim, nCs, tess, prec)
        np_dt = np.float64 if prec == torch.float64 else np.float32
        sizes = [int(np.asarray(r.req.pts).shape[0]) for r in recs]
        offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        total = int(offs[-1])
        tdt = torch.float64 if np_dt == np.float64 else torch.float32
        pin_x = self._pinned_buf(total * dim, tdt)
        pin_o = self._pinned_buf(total * dim, tdt)
        pin_th = self._pinned_buf(len(recs) * sp.d, torch.float64)
        pin_off = self._pinned_buf(len(offs), torch.int64)
        xv = pin_x[:total * dim].numpy().reshape(total, dim)
        for r, a, b in zip(recs, offs[:-1], offs[1:]):
            xv[a:b] = np.asarray(r.req.pts, dtype=np_dt).reshape(-1, dim)
        pin_th[:len(recs) * sp.d].numpy().reshape(len(recs), sp.d)[:] = np.stack(
            [np.asarray(r.req.theta, dtype=np.float64) for r in recs])
        pin_off[:len(offs)].numpy()[:] = offs
        stream = self.streams[next(self._rr)]
        sch = {"exact": _lib.SCHEME_EXACT, "ref": _lib.SCHEME_REF, "simple": _lib.SCHEME_SIMPLE}[scheme]
        with torch.cuda.stream(stream):
            x = pin_x[:total * dim].view(total, dim).to(self.device, non_blocking=True)
            th = pin_th[:len(recs) * sp.d].view(len(recs), sp.d).to(self.device, non_blocking=True)
            off = pin_off[:len(offs)].to(self.device, non_blocking=True)
            out = torch.empty_like(x)
            tables = sp.tables_from_theta(th, float(params["dt"]), sign)
            sp.calc_T_batched(tables, x, out, offsets=off, scheme=sch, **params)
            pin_o[:total * dim].view(total, dim).copy_(out, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        keep = (x, th, off, out, tables)            # device buffers live until retired

        def finalize(recs=recs, offs=offs, keep=keep, bufs=(pin_x, pin_o, pin_th, pin_off), total=total):
            res = bufs[1][:total * dim].numpy().reshape(total, dim)
            for r, a, b in zip(recs, offs[:-1], offs[1:]):
                r.result = res[a:b].copy()
            self._release_pinned(*bufs)
        self.inflight.append((ev, recs, finalize))

    def _start_job(self, r: _Record) -> None:
        q: RegistrationRequest = r.req
        sp = self.space(2, q.nCs, q.tess, torch.float32, for_jobs=True)
        stream = self.job_streams[next(self._rr_jobs)]
        with torch.cuda.stream(stream):
            src = torch.as_tensor(np.asarray(q.src, dtype=np.float32), device=self.device)
            dst = torch.as_tensor(np.asarray(q.dst, dtype=np.float32), device=self.device)
            ll = GaussianLogLikelihood(sp, src, dst, q.sigma, params_flow_int=q.params)
            prop_std = np.sqrt(np.diag(self.prior(sp).cov_cpa))
            mh = BatchedMetropolis(ll, torch.zeros((1, sp.d), dtype=torch.float64, device=self.device), prop_std,
                                   scale=q.scale, seed=q.seed, rule=q.rule)
        self.jobs.append(dict(rec=r, mh=mh, stream=stream, left=int(q.n_steps), keep=(src, dst), ev=None))

    def _advance_jobs(self) -> None:
        running = []
        for job in self.jobs:
            if job["ev"] is not None and not job["ev"].query():
                running.append(job)            # one slice in flight per job
                continue
            k = min(self.mcmc_slice, job["left"])
            with torch.cuda.stream(job["stream"]):
                mh = job["mh"]
                if k == self.mcmc_slice and job.get("warm"):
                    # full slices replay a CUDA graph captured on this stream (one host call per slice)
                    if mh._graph is None:
                        mh.capture(self.mcmc_slice)
                    mh._graph.replay()
                else:
                    mh.run(k)
                    job["warm"] = True
                job["left"] -= k
                if job["left"] == 0:
                    mh = job["mh"]
                    th_h = torch.empty_like(mh.theta, device="cpu").pin_memory()
                    ll_h = torch.empty_like(mh.ll, device="cpu").pin_memory()
                    acc_h = torch.empty_like(mh.n_accepted, device="cpu").pin_memory()
                    th_h.copy_(mh.theta, non_blocking=True)
                    ll_h.copy_(mh.ll, non_blocking=True)
                    acc_h.copy_(mh.n_accepted, non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(job["stream"])

                    def finalize(rec=job["rec"], th_h=th_h, ll_h=ll_h, acc_h=acc_h, keep=(mh, job["keep"])):
                        rec.result = dict(theta=th_h.numpy()[0].copy(), ll=float(ll_h[0]),
                                          accepted=int(acc_h[0]))
                    self.inflight.append((ev, [job["rec"]], finalize))
                else:
                    job["ev"] = torch.cuda.Event()
                    job["ev"].record(job["stream"])
                    running.append(job)
        self.jobs = running
