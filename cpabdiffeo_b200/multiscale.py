"""Coarse-to-fine multiscale spaces and batched multiscale registration.

Mirrors
  * cpab/cpaNd/_Multiscale.py:139-292: a pyramid of CPA spaces whose
    tessellation is refined by 2 per axis from one level to the next, and
    propogate_theta_coarse2fine: A_coarse = B_coarse theta_coarse, every fine
    cell takes the affine map of the coarse cell that contains it
    (propogate_Avees_coarser2fine), theta_fine = B_fine^T A_fine
    (Avees2theta, cpab/cpaNd/_CpaSpace.py:377-390).  The fine tessellations
    are nested in the coarse ones, so a continuous coarse field is also a
    continuous fine field and the projection reproduces it exactly.
  * cpab/cpa2d/inference/transformation/Register.py:171-287 (Register.fit):
    for each level, start from the propagated theta, run Metropolis for that
    level's run length with the coarse integration parameters, propagate.
    Here C chains (one image pair each) run in lock-step on the GPU per level
    (BatchedMetropolis, graph-captured steps).
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from .cpa_space import CpaSpace
from .mcmc import BatchedMetropolis
from .registration import GaussianLogLikelihood
from .space import Prior, SpaceGeometry


def _inside(cells: np.ndarray, pts: np.ndarray, tess: str, tol: float = 1e-9) -> np.ndarray:
    """Boolean [nPts, nC]: point inside (or on the boundary of) each cell."""
    dim = pts.shape[1]
    V = cells[:, :, :dim]
    if tess == "II" or dim == 1:
        lo, hi = V.min(axis=1), V.max(axis=1)
        return np.all((pts[:, None, :] >= lo[None] - tol) & (pts[:, None, :] <= hi[None] + tol), axis=2)
    # simplices: barycentric coordinates of every point in every cell
    T = V[:, 1:, :] - V[:, :1, :]                         # [nC, dim, dim] edge vectors (rows)
    Tinv = np.linalg.inv(np.transpose(T, (0, 2, 1)))      # [nC, dim, dim]
    rel = pts[:, None, :] - V[None, :, 0, :]              # [nPts, nC, dim]
    lam = np.einsum("cij,pcj->pci", Tinv, rel)            # [nPts, nC, dim]
    lam0 = 1.0 - lam.sum(axis=2)
    return np.all(lam >= -tol, axis=2) & (lam0 >= -tol)


def parent_cells(coarse: SpaceGeometry, fine: SpaceGeometry) -> np.ndarray:
    """For every fine cell, the coarse cell that contains it (int64 [nC_fine]).
    Raises NotImplementedError when some fine cell is not inside one coarse cell
    (the reference does not propagate 3D type-I tessellations either,
    cpab/cpaNd/_Multiscale.py:259-262)."""
    dim = fine.dim
    cen = fine.cells[:, :, :dim].mean(axis=1)
    par = np.argmax(_inside(coarse.cells, cen, coarse.tess), axis=1)
    # every vertex of a fine cell must lie in its parent
    nV = fine.cells.shape[1]
    verts = fine.cells[:, :, :dim].reshape(-1, dim)
    ok = _inside(coarse.cells, verts, coarse.tess)[np.arange(verts.shape[0]), np.repeat(par, nV)]
    if not ok.all():
        raise NotImplementedError("the fine tessellation is not nested in the coarse one")
    return par.astype(np.int64)


class Multiscale:
    """L_cpa_space[level]: the CPA space of `base * 2**level` cells per axis on
    the domain [XMINS, XMAXS] (cpab/cpaNd/_Multiscale.py)."""

    def __init__(self, XMINS: Sequence[float], XMAXS: Sequence[float], base: Sequence[int], nLevels: int,
                 tess: str = "II", zero_v_across_bdry: Sequence[bool] | None = None, device=None,
                 precision: torch.dtype = torch.float64):
        if nLevels < 1:
            raise ValueError(nLevels)
        self.nLevels = int(nLevels)
        self.dim_domain = len(base)
        self.L_cpa_space = [CpaSpace(XMINS, XMAXS, tuple(int(b) * 2 ** lev for b in base), tess=tess,
                                     zero_v_across_bdry=zero_v_across_bdry, device=device, precision=precision)
                            for lev in range(self.nLevels)]
        self._parents = {}

    def parents(self, level_coarse: int) -> torch.Tensor:
        if level_coarse not in self._parents:
            sc, sf = self.L_cpa_space[level_coarse], self.L_cpa_space[level_coarse + 1]
            self._parents[level_coarse] = torch.as_tensor(parent_cells(sc.geo, sf.geo), device=sf.device)
        return self._parents[level_coarse]

    def propagate_theta_coarse2fine(self, theta_coarse: torch.Tensor, level_coarse: int) -> torch.Tensor:
        """theta [C, d_coarse] (or [d_coarse]) at level_coarse -> theta [C, d_fine] at level_coarse + 1."""
        sc, sf = self.L_cpa_space[level_coarse], self.L_cpa_space[level_coarse + 1]
        th = torch.as_tensor(theta_coarse, dtype=torch.float64, device=sc.device)
        one = th.ndim == 1
        th = th.reshape(-1, sc.d)
        ne = sc.geo.lengthAvee
        A_c = (th @ sc.B.T).reshape(th.shape[0], sc.nC, ne)        # A = B theta, per chain
        A_f = A_c[:, self.parents(level_coarse), :].reshape(th.shape[0], sf.D)
        th_f = A_f @ sf.B                                          # theta = B^T A
        return th_f[0] if one else th_f

    # the reference's spelling
    propogate_theta_coarse2fine = propagate_theta_coarse2fine


class MultiscaleRegister:
    """Batched coarse-to-fine registration of C image pairs (2D, unit square):
    per level a Gaussian likelihood on that level's space, C Metropolis chains
    started from the propagated theta (Register.fit, cpab/cpa2d/inference/
    transformation/Register.py:171-287)."""

    def __init__(self, ms: Multiscale, src: torch.Tensor, dst: torch.Tensor, sigma_signal: float,
                 params_flow_int: dict, proposal_scale: float = 0.05, length_scale: float = 0.1,
                 variance: float = 1.0, seed: int = 0, rule: str = "reference"):
        if ms.dim_domain != 2:
            raise ValueError("2D images")
        self.ms = ms
        self.src = src if src.ndim == 3 else src.unsqueeze(0)
        self.dst = dst if dst.ndim == 3 else dst.unsqueeze(0)
        self.C = self.src.shape[0]
        self.sigma = float(sigma_signal)
        self.params = dict(params_flow_int)
        self.scale = float(proposal_scale)
        self.length_scale, self.variance = float(length_scale), float(variance)
        self.seed = int(seed)
        self.rule = rule
        self.records: list[dict] = []

    def fit(self, run_lengths: Sequence[int], graph_steps: int = 0) -> torch.Tensor:
        """Runs every level; returns theta [C, d] of the finest level."""
        if len(run_lengths) != self.ms.nLevels:
            raise ValueError(len(run_lengths), self.ms.nLevels)
        theta = None
        self.records = []
        for level, n_steps in enumerate(run_lengths):
            sp = self.ms.L_cpa_space[level]
            if level == 0:
                theta = torch.zeros((self.C, sp.d), dtype=torch.float64, device=sp.device)
            else:
                theta = self.ms.propagate_theta_coarse2fine(theta, level - 1)
            prior = Prior.create(sp.geo, self.length_scale, self.variance)
            ll = GaussianLogLikelihood(sp, self.src, self.dst, self.sigma, self.params)
            mh = BatchedMetropolis(ll, theta, np.sqrt(np.diag(prior.cov_cpa)), scale=self.scale,
                                   seed=self.seed + level, rule=self.rule)
            ll0 = mh.ll.clone()
            if n_steps > 0:
                gs = min(graph_steps, n_steps) if graph_steps > 0 else 0
                mh.run(int(n_steps), graph_steps=gs)
            theta = mh.theta.clone()
            self.records.append(dict(level=level, d=sp.d, nC=sp.nC, steps=int(n_steps), ll_start=ll0,
                                     ll_end=mh.ll.clone(), accept_pct=mh.accept_ratio()))
        return theta
