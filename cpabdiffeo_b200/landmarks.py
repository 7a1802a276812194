"""Gaussian landmark log-likelihood, batched over theta, on torch CUDA tensors.

Mirrors ScaleDependentLogLikelihoodGaussian of
cpab/cpa2d/model/transformations/landmarks/_ScaleDependentLogLikelihoodGaussian.py
(calc_ll :29-73, gpu/gaussian.py:12-22) and its 1D twin
cpab/cpa1d/model/transformations/landmarks/:

    ll_i(theta) = -0.5 |T_theta(src_i) - dst_i|^2 / sigma_lm^2,   T = calc_T_fwd

and __call__ (cpab/cpa2d/.../_ScaleDependentLogLikelihoodGeneral.py:80-113
returns the mean over landmarks; cpab/cpa1d/.../_ScaleDependentLogLikelihoodGeneral.py:71-88
returns the sum).  One fused launch integrates every landmark of every theta
and reduces each theta's terms in a fixed order (cpab_landmark_ll).
"""
from __future__ import annotations

import torch

from . import _lib
from .cpa_space import CpaSpace, default_params_flow_int


class LandmarkLogLikelihood:
    """src, dst: landmarks [n_lm, dim] shared by every theta, or [N, n_lm, dim]
    (one set per theta; N fixed at construction).  float64 on the space's device.
    n_theta: the batch size reported as N (the number of chains a
    BatchedMetropolis runs) when the landmark set is shared."""

    sign = 1              # landmarks are pushed forward: calc_T_fwd

    def __init__(self, space: CpaSpace, src: torch.Tensor, dst: torch.Tensor, sigma_lm: float,
                 params_flow_int: dict | None = None, precision: torch.dtype | None = None,
                 n_theta: int | None = None):
        dev = space.device
        src = torch.as_tensor(src, dtype=torch.float64, device=dev).contiguous()
        dst = torch.as_tensor(dst, dtype=torch.float64, device=dev).contiguous()
        if src.shape != dst.shape or src.shape[-1] != space.dim or src.ndim not in (2, 3):
            raise ValueError(f"src/dst must be [n_lm, {space.dim}] or [N, n_lm, {space.dim}], got "
                             f"{tuple(src.shape)} / {tuple(dst.shape)}")
        self.space = space
        self.src, self.dst = src, dst
        self.shared = src.ndim == 2
        self.n_lm = int(src.shape[-2])
        if self.n_lm < 1:
            raise ValueError("at least one landmark")
        self.N = (int(n_theta) if n_theta else 1) if self.shared else int(src.shape[0])
        self.nPts = self.n_lm
        self.sigma = float(sigma_lm)
        p = default_params_flow_int(space.dim)
        if params_flow_int:
            p.update(params_flow_int)
        self.dt, self.nT, self.nODE = float(p["dt"]), int(p["nTimeSteps"]), int(p["nStepsODEsolver"])
        self.prec = _lib.CPAB_F64 if (precision or space.precision) == torch.float64 else _lib.CPAB_F32
        self._ws = {}
        self.nCalls = 0

    def _workspace(self, N: int) -> torch.Tensor:
        if N not in self._ws:
            c = self.space._ctx
            nb = c.lib.cpab_landmark_workspace_bytes(c.h, N, self.n_lm)
            self._ws[N] = torch.empty(max(int(nb), 1), dtype=torch.uint8, device=self.space.device)
        return self._ws[N]

    def batch(self, theta: torch.Tensor, transformed: torch.Tensor | None = None,
              counters: torch.Tensor | None = None) -> torch.Tensor:
        """Sum over landmarks of ll_i for theta [N, d] (any N when the landmark
        set is shared), float64 [N]; transformed [N, n_lm, dim] float64 receives
        T_theta(src) when given."""
        th = torch.as_tensor(theta, dtype=torch.float64, device=self.space.device)
        th = th.reshape(-1, self.space.d)
        return self.batch_tables(self.space.tables_from_theta(th, self.dt, 1), transformed=transformed,
                                 counters=counters)

    def batch_tables(self, tables, transformed=None, counters=None, ll=None) -> torch.Tensor:
        sA, Tr = tables
        N = int(sA.shape[0])
        if not self.shared and N != self.N:
            raise ValueError(f"{self.N} landmark sets for {N} thetas")
        if transformed is not None and (tuple(transformed.shape) != (N, self.n_lm, self.space.dim)
                                        or transformed.dtype != torch.float64 or not transformed.is_contiguous()):
            raise ValueError("transformed must be contiguous float64 [N, n_lm, dim]")
        ll = torch.empty(N, dtype=torch.float64, device=self.space.device) if ll is None else ll
        stride = 0 if self.shared else self.n_lm
        ws = self._workspace(N)
        c = self.space._ctx
        c.check(c.lib.cpab_landmark_ll(c.h, _lib.ptr(sA), _lib.ptr(Tr), N, _lib.ptr(self.src), stride,
                                       _lib.ptr(self.dst), stride, self.n_lm, self.sigma, self.prec, self.dt,
                                       self.nT, self.nODE, _lib.ptr(ll), _lib.ptr(transformed), _lib.ptr(ws),
                                       ws.numel(), _lib.ptr(counters), _lib.stream_ptr()))
        return ll

    def __call__(self, theta) -> float:
        """The reference's value for one theta: the mean over landmarks in 2D/3D
        (cpa2d __call__), the sum in 1D (cpa1d __call__)."""
        self.nCalls += 1
        s = float(self.batch(torch.as_tensor(theta).reshape(1, -1))[0].item())
        return s if self.space.dim == 1 else s / self.n_lm
