"""Batched Metropolis-Hastings registration: C independent chains, each with
its own data (an image pair, a volume pair or a landmark set), advanced in
lock-step on the GPU.

One step per chain (cpab/cpaNd/inference/Metropolis.py:41-85,
cpab/cpaNd/inference/Proposal.py:29-130):
  theta' = theta + scale * sqrt(diag Sigma_CPA) * z   (random walk), or the
           local proposal: one vertex velocity perturbed (use_local=True)
  ll'    = log-likelihood of theta' (fused kernel, map never stored)
  log_ratio = (ll' - ll) / nPts  [+ wlp * (lp' - lp)]
  accept if log_ratio > 0, else by u ~ U(0,1) with the reference's own test
  log(u) > log_ratio (rule="reference", the default) or the textbook test
  log(u) < log_ratio (rule="standard").
State (theta, ll, lp, acceptance counts, the step counter) stays on the GPU;
several steps can be captured in one CUDA graph and replayed.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .cpa_space import CpaSpace


class BatchedMetropolis:
    def __init__(self, ll, theta0: torch.Tensor, prop_std: np.ndarray | None = None, scale: float = 0.05,
                 seed: int = 0, rule: str = "reference", use_ave_ll: bool = True,
                 prior_precision: np.ndarray | None = None, wlp: float = 1.0, use_local: bool = False,
                 scale_local_proposal: float = 10.0):
        """ll: GaussianLogLikelihood(3D) or LandmarkLogLikelihood.  use_local
        selects the local (vertex-velocity) proposal of Proposal.py:65-130 with
        step scale_local_proposal * min(XMAXS) (0.01 in 1D, :96-103) instead of
        the Gaussian random walk with prop_std."""
        self.ll_fn = ll
        sp: CpaSpace = ll.space
        self.space = sp
        dev = sp.device
        # image likelihoods integrate with calc_T_inv tables, landmark ones with calc_T_fwd
        self.sign = int(getattr(ll, "sign", -1))
        self.C = ll.N
        self.d = sp.d
        self.theta = torch.as_tensor(theta0, dtype=torch.float64, device=dev).reshape(self.C, self.d).clone()
        self.theta_prop = torch.empty_like(self.theta)
        self.use_local = bool(use_local)
        if self.use_local:
            from .space import local_proposal_tables
            tabs = local_proposal_tables(sp.geo)
            self.local_nV = int(tabs.vertices.shape[0])
            self.local_E = torch.as_tensor(tabs.E, device=dev).contiguous()
            self.local_G = torch.as_tensor(tabs.G, device=dev).contiguous()
            self.local_bdry = torch.as_tensor(tabs.bdry.astype(np.int32), device=dev).contiguous()
            self.local_s = float(scale_local_proposal) * float(np.min(sp.XMAXS)) if sp.dim > 1 else 0.01
            self.prop_std = None
        else:
            if prop_std is None:
                raise ValueError("prop_std is needed for the random-walk proposal")
            if isinstance(prop_std, torch.Tensor) and prop_std.is_cuda:
                # already resident (a server shares one per space): no host copy, no stream sync
                self.prop_std = prop_std.to(device=dev, dtype=torch.float64).contiguous()
            else:
                self.prop_std = torch.as_tensor(np.asarray(prop_std, dtype=np.float64), device=dev).contiguous()
        self.scale = float(scale)
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.rule = {"reference": 0, "standard": 1}[rule]
        self.inv_npts = 1.0 / ll.nPts if use_ave_ll else 1.0
        self.prior_prec = (torch.as_tensor(prior_precision, dtype=torch.float64, device=dev).contiguous()
                           if prior_precision is not None else None)
        self.wlp = float(wlp)
        self.step = torch.zeros(1, dtype=torch.int64, device=dev)
        self.n_accepted = torch.zeros(self.C, dtype=torch.int64, device=dev)
        self.ll_prop = torch.empty(self.C, dtype=torch.float64, device=dev)
        D = sp.D
        self.sA = torch.empty((self.C, D), dtype=torch.float64, device=dev)
        self.Tr = torch.empty_like(self.sA)
        # current likelihood and prior
        self.ll = ll.batch(self.theta).clone()
        self.lp = None
        if self.prior_prec is not None:
            th = self.theta
            self.lp = -0.5 * torch.einsum("ci,ij,cj->c", th, self.prior_prec, th)
        self._graph = None
        self._graph_steps = 0

    def _step_launches(self) -> None:
        sp, c = self.space, self.space._ctx
        s = _lib.stream_ptr()
        if self.use_local:
            c.check(c.lib.cpab_mcmc_propose_local(c.h, self.C, self.d, _lib.ptr(self.theta), self.local_nV,
                                                  _lib.ptr(self.local_E), _lib.ptr(self.local_G),
                                                  _lib.ptr(self.local_bdry), self.local_s, self.seed,
                                                  _lib.ptr(self.step), _lib.ptr(self.theta_prop), s))
        else:
            c.check(c.lib.cpab_mcmc_propose(c.h, self.C, self.d, _lib.ptr(self.theta), _lib.ptr(self.prop_std),
                                            self.scale, self.seed, _lib.ptr(self.step), _lib.ptr(self.theta_prop), s))
        c.check(c.lib.cpab_theta_to_trels(c.h, _lib.ptr(sp.B), self.d, _lib.ptr(self.theta_prop), self.C,
                                          self.ll_fn.dt, self.sign, None, _lib.ptr(self.sA), _lib.ptr(self.Tr), s))
        self.ll_fn.batch_tables((self.sA, self.Tr), ll=self.ll_prop)
        c.check(c.lib.cpab_mcmc_accept(c.h, self.C, self.d, _lib.ptr(self.theta), _lib.ptr(self.theta_prop),
                                       _lib.ptr(self.ll), _lib.ptr(self.ll_prop), self.inv_npts,
                                       _lib.ptr(self.prior_prec), self.wlp, _lib.ptr(self.lp), self.rule, self.seed,
                                       _lib.ptr(self.step), _lib.ptr(self.n_accepted), s))

    def capture(self, graph_steps: int) -> None:
        """Capture `graph_steps` steps into a CUDA graph on the current stream
        without a device-wide synchronisation (for servers that keep other
        streams busy).  Needs one eager step beforehand; allocates nothing."""
        g = torch.cuda.CUDAGraph()
        g.capture_begin(capture_error_mode="thread_local")
        try:
            for _ in range(graph_steps):
                self._step_launches()
        finally:
            g.capture_end()
        self._graph, self._graph_steps = g, graph_steps

    def run(self, n_steps: int, graph_steps: int = 0) -> None:
        """Advance every chain by n_steps.  graph_steps > 0 captures that many
        steps in a CUDA graph (once) and replays it; the remainder runs eagerly."""
        if graph_steps <= 0:
            for _ in range(n_steps):
                self._step_launches()
            return
        if self._graph is None or self._graph_steps != graph_steps:
            # make sure every kernel attribute is set before capture
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            saved = (self.theta.clone(), self.ll.clone(), self.step.clone(), self.n_accepted.clone(),
                     None if self.lp is None else self.lp.clone())
            with torch.cuda.graph(g):
                for _ in range(graph_steps):
                    self._step_launches()
            # capture does not execute; restore to be safe
            self.theta.copy_(saved[0]); self.ll.copy_(saved[1]); self.step.copy_(saved[2])
            self.n_accepted.copy_(saved[3])
            if self.lp is not None:
                self.lp.copy_(saved[4])
            self._graph, self._graph_steps = g, graph_steps
        for _ in range(n_steps // graph_steps):
            self._graph.replay()
        for _ in range(n_steps % graph_steps):
            self._step_launches()

    def accept_ratio(self) -> np.ndarray:
        """Percentage of accepted proposals per chain (Metropolis.py:84-85)."""
        steps = int(self.step.item())
        return self.n_accepted.cpu().numpy() * 100.0 / max(steps, 1)
