"""Differentiable CPAB transforms: torch.autograd.Function over the adjoint
kernel (cpab_grad_theta).

    y = transform(theta, pts, space, dt=..., nTimeSteps=..., nStepsODEsolver=...)
    loss = 0.5 * ((y - target) ** 2).sum();  loss.backward()   # theta.grad

scheme="ref" (default): the forward is calc_T, the reference scheme
(closed-form steps T = expm(dt A), nStepsODE midpoint sub-steps where a step
leaves its cell); the backward (cpab_grad_theta_ref) re-runs it with
checkpoints every `ck` time steps and propagates dLoss/dT(x) back through
every step along the branch the forward took, mapping the per-cell
dLoss/dT to dLoss/dA through the adjoint Frechet derivative of expm.
scheme="simple": the forward is calc_T_simple (nTimeSteps * nStepsODE
midpoint sub-steps) and the backward (cpab_grad_theta) goes through every
sub-step.  Either is the exact gradient of the discrete map.  theta is
[N, d] float64 (N transforms), pts [N*n, dim] (n points per transform)
float64, or float32 with scheme="ref" (the FP32 calc_T and its adjoint; the
gradient in theta comes back float64).
"""
from __future__ import annotations

import torch

from . import _lib
from .cpa_space import CpaSpace, default_params_flow_int


def _flow(space: CpaSpace, params: dict):
    p = default_params_flow_int(space.dim)
    p.update(params)
    return float(p["dt"]), int(p["nTimeSteps"]), int(p["nStepsODEsolver"])


def checkpoint_stride(space: CpaSpace, N: int, n: int, nT: int, budget_bytes: int) -> int:
    """Smallest checkpoint stride whose scratch fits in budget_bytes (recompute
    trajectories rather than store them when memory asks)."""
    per_ck = N * n * space.dim * 8
    for ck in range(1, nT + 1):
        if -(-nT // ck) * per_ck <= budget_bytes:
            return ck
    return nT


class _Transform(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, pts, space, sign, dt, nT, nODE, ck, need_pts_grad, ref):
        N = theta.shape[0]
        n = pts.shape[0] // N
        sA, Tr = space.tables_from_theta(theta.detach(), dt, sign)
        out = torch.empty_like(pts)
        c = space._ctx
        prec = _lib.CPAB_F64 if pts.dtype == torch.float64 else _lib.CPAB_F32
        c.check(c.lib.cpab_calc_T_batched(c.h, _lib.ptr(sA), _lib.ptr(Tr), _lib.ptr(pts), _lib.ptr(out), N, None, n,
                                          None, 0, prec, _lib.SCHEME_REF if ref else _lib.SCHEME_SIMPLE,
                                          dt, nT, nODE, None, _lib.stream_ptr()))
        ctx.save_for_backward(pts, sA, Tr)
        ctx.space, ctx.sign, ctx.dt, ctx.nT, ctx.nODE, ctx.ck = space, sign, dt, nT, nODE, ck
        ctx.need_pts_grad, ctx.ref = need_pts_grad, ref
        return out

    @staticmethod
    def backward(ctx, grad_out):
        pts, sA, Tr = ctx.saved_tensors
        sp: CpaSpace = ctx.space
        N = sA.shape[0]
        n = pts.shape[0] // N
        g = grad_out.contiguous().to(pts.dtype)
        prec = _lib.CPAB_F64 if pts.dtype == torch.float64 else _lib.CPAB_F32
        dtheta = torch.empty((N, sp.d), dtype=torch.float64, device=pts.device)
        gA = torch.empty((N, sp.D), dtype=torch.float64, device=pts.device)
        gpts = torch.empty_like(pts) if ctx.need_pts_grad else None
        c = sp._ctx
        if ctx.ref:
            wsb = int(c.lib.cpab_grad_ref_workspace_bytes(c.h, N, n, ctx.nT, ctx.ck))
            ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=pts.device)
            c.check(c.lib.cpab_grad_theta_ref(c.h, _lib.ptr(sp.B), sp.d, _lib.ptr(sA), _lib.ptr(Tr), N, _lib.ptr(pts),
                                              n, _lib.ptr(g), prec, ctx.dt, ctx.nT, ctx.nODE, ctx.sign, ctx.ck, None,
                                              _lib.ptr(gpts), _lib.ptr(gA), _lib.ptr(dtheta), _lib.ptr(ws),
                                              ws.numel(), _lib.stream_ptr()))
        else:
            wsb = int(c.lib.cpab_grad_workspace_bytes(c.h, N, n, ctx.nT, ctx.ck))
            ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=pts.device)
            c.check(c.lib.cpab_grad_theta(c.h, _lib.ptr(sp.B), sp.d, _lib.ptr(sA), N, _lib.ptr(pts), n, _lib.ptr(g),
                                          ctx.dt, ctx.nT, ctx.nODE, ctx.sign, ctx.ck, None, _lib.ptr(gpts),
                                          _lib.ptr(gA), _lib.ptr(dtheta), _lib.ptr(ws), ws.numel(),
                                          _lib.stream_ptr()))
        return dtheta, gpts, None, None, None, None, None, None, None, None


def transform(theta: torch.Tensor, pts: torch.Tensor, space: CpaSpace, mysign: int = 1, ck: int | None = None,
              memory_budget_bytes: int = 8 << 30, scheme: str = "ref", **params_flow_int) -> torch.Tensor:
    """T_theta(pts) (or T^-1 with mysign=-1), differentiable in theta and pts, through the reference
    scheme (calc_T, scheme="ref") or the midpoint scheme (calc_T_simple, scheme="simple")."""
    if scheme not in ("ref", "simple"):
        raise ValueError('scheme must be "ref" or "simple"')
    dt, nT, nODE = _flow(space, params_flow_int)
    theta = theta.reshape(-1, space.d)
    if theta.dtype != torch.float64:
        raise TypeError("theta must be float64")
    if pts.dtype != torch.float64 and not (pts.dtype == torch.float32 and scheme == "ref"):
        raise TypeError("pts must be float64 (or float32 with scheme='ref')")
    N = theta.shape[0]
    if pts.shape[0] % N:
        raise ValueError("pts must hold the same number of points for every theta")
    if ck is None:
        ck = checkpoint_stride(space, N, pts.shape[0] // N, nT, memory_budget_bytes)
    return _Transform.apply(theta, pts.contiguous(), space, int(mysign), dt, nT, nODE, int(ck),
                            bool(pts.requires_grad), scheme == "ref")
