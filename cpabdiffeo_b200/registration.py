"""Image-side API: remap, TransformWrapper (2D), and the Gaussian registration
log-likelihood, on torch CUDA tensors.

Mirrors
  * cpab/cpa2d/TransformWrapper.py (calc_T_fwd/inv, calc_v, calc_trajectory,
    calc_cell_idx, remap_fwd / remap_inv :261-317) on the reference's pixel
    domain [0, nCols] x [0, nRows] with points at integer pixel coordinates;
  * cpab/cpa2d/model/transformations/register/_ScaleDependentLogLikelihoodGaussian.py
    (calc_ll :34-109) and _ScaleDependentLogLikelihoodGeneral.__call__
    (:108-131): ll(theta) = sum_i -0.5 (src(T^-1 x_i) - dst(x_i))^2 / sigma^2,
    here on the unit square with pixel centres at ((c+0.5)/W, (r+0.5)/H),
    for one theta or a batch of thetas (one fused launch).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .cpa_space import CpaSpace, default_params_flow_int

_MAP_DT = {torch.float64: _lib.CPAB_F64, torch.float32: _lib.CPAB_F32}


def _ws(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def remap(map_pts: torch.Tensor, img: torch.Tensor, out: torch.Tensor | None = None,
          pixel_map=(1.0, 0.0, 1.0, 0.0)) -> torch.Tensor:
    """out[i] = bilinear(img, map_pts[i]) with cv2.remap semantics (zero outside).
    map_pts [H*W, 2] (or [N, H*W, 2]), img [H, W] (or [N, H, W]) float32.
    pixel_map = (sx, ox, sy, oy): a map point (x, y) is sampled at pixel
    coordinates (x*sx + ox, y*sy + oy)."""
    lib = _lib.load()
    imgs = img if img.ndim == 3 else img.unsqueeze(0)
    N, H, W = imgs.shape
    if imgs.dtype != torch.float32 or not imgs.is_contiguous():
        raise ValueError("images must be contiguous float32")
    mp = map_pts if map_pts.ndim == 3 else map_pts.unsqueeze(0)
    if tuple(mp.shape) != (N, H * W, 2) or mp.dtype not in _MAP_DT or not mp.is_contiguous():
        raise ValueError(f"map must be contiguous [N, H*W, 2] float32/float64, got {tuple(mp.shape)} {mp.dtype}")
    if out is None:
        out = torch.zeros_like(imgs)
    sx, ox, sy, oy = pixel_map
    _lib.check(lib.cpab_remap_ssd(None, _lib.ptr(mp), _MAP_DT[mp.dtype], _lib.ptr(imgs), None, N, H, W,
                                  float(sx), float(ox), float(sy), float(oy), 1.0, _lib.ptr(out), None, None, 0,
                                  _lib.stream_ptr()))
    return out if img.ndim == 3 else out[0]


def remap_ssd(map_pts: torch.Tensor, src: torch.Tensor, dst: torch.Tensor, sigma: float,
              pixel_map=(1.0, 0.0, 1.0, 0.0), warped: torch.Tensor | None = None) -> torch.Tensor:
    """ll[n] = sum -0.5 (bilinear(src[n], map[n]) - dst[n])^2 / sigma^2, float64 [N]."""
    lib = _lib.load()
    srcs = src if src.ndim == 3 else src.unsqueeze(0)
    dsts = dst if dst.ndim == 3 else dst.unsqueeze(0)
    N, H, W = srcs.shape
    mp = map_pts if map_pts.ndim == 3 else map_pts.unsqueeze(0)
    if dsts.shape != srcs.shape or srcs.dtype != torch.float32 or dsts.dtype != torch.float32:
        raise ValueError("src/dst must be float32 images of the same shape")
    if tuple(mp.shape) != (N, H * W, 2) or mp.dtype not in _MAP_DT:
        raise ValueError("map must be [N, H*W, 2]")
    ll = torch.empty(N, dtype=torch.float64, device=srcs.device)
    ws = _ws(lib.cpab_remap_workspace_bytes(N, H, W), srcs.device)
    sx, ox, sy, oy = pixel_map
    _lib.check(lib.cpab_remap_ssd(None, _lib.ptr(mp.contiguous()), _MAP_DT[mp.dtype], _lib.ptr(srcs.contiguous()),
                                  _lib.ptr(dsts.contiguous()), N, H, W, float(sx), float(ox), float(sy), float(oy),
                                  float(sigma), _lib.ptr(warped), _lib.ptr(ll), _lib.ptr(ws), ws.numel(),
                                  _lib.stream_ptr()))
    return ll


def remap3d(map_pts: torch.Tensor, vol: torch.Tensor, out: torch.Tensor | None = None,
            voxel_map=(1.0, 0.0, 1.0, 0.0, 1.0, 0.0)) -> torch.Tensor:
    """out[i] = trilinear(vol, map_pts[i]), zero outside (remap3d of
    cpab/cpa3d/TransformWrapper.py:254-286).  vol [H, W, D] (or [N, H, W, D])
    float32 indexed [row][col][slice]; map_pts [H*W*D, 3] (or [N, H*W*D, 3])
    points (x, y, z) = (column, row, slice); voxel_map = (sx, ox, sy, oy, sz, oz)
    samples a point at voxel coordinates (x*sx + ox, y*sy + oy, z*sz + oz)."""
    lib = _lib.load()
    vols = vol if vol.ndim == 4 else vol.unsqueeze(0)
    N, H, W, D = vols.shape
    if vols.dtype != torch.float32 or not vols.is_contiguous():
        raise ValueError("volumes must be contiguous float32")
    mp = map_pts if map_pts.ndim == 3 else map_pts.unsqueeze(0)
    if tuple(mp.shape) != (N, H * W * D, 3) or mp.dtype not in _MAP_DT or not mp.is_contiguous():
        raise ValueError(f"map must be contiguous [N, H*W*D, 3] float32/float64, got {tuple(mp.shape)} {mp.dtype}")
    if out is None:
        out = torch.zeros_like(vols)
    _lib.check(lib.cpab_remap3d_ssd(None, _lib.ptr(mp), _MAP_DT[mp.dtype], _lib.ptr(vols), None, N, H, W, D,
                                    *map(float, voxel_map), 1.0, _lib.ptr(out), None, None, 0, _lib.stream_ptr()))
    return out if vol.ndim == 4 else out[0]


def remap3d_ssd(map_pts: torch.Tensor, src: torch.Tensor, dst: torch.Tensor, sigma: float,
                voxel_map=(1.0, 0.0, 1.0, 0.0, 1.0, 0.0), warped: torch.Tensor | None = None) -> torch.Tensor:
    """ll[n] = sum -0.5 (trilinear(src[n], map[n]) - dst[n])^2 / sigma^2, float64 [N]."""
    lib = _lib.load()
    srcs = src if src.ndim == 4 else src.unsqueeze(0)
    dsts = dst if dst.ndim == 4 else dst.unsqueeze(0)
    N, H, W, D = srcs.shape
    mp = map_pts if map_pts.ndim == 3 else map_pts.unsqueeze(0)
    if dsts.shape != srcs.shape or srcs.dtype != torch.float32 or dsts.dtype != torch.float32:
        raise ValueError("src/dst must be float32 volumes of the same shape")
    if tuple(mp.shape) != (N, H * W * D, 3) or mp.dtype not in _MAP_DT:
        raise ValueError("map must be [N, H*W*D, 3]")
    ll = torch.empty(N, dtype=torch.float64, device=srcs.device)
    ws = _ws(lib.cpab_remap3d_workspace_bytes(N, H, W, D), srcs.device)
    _lib.check(lib.cpab_remap3d_ssd(None, _lib.ptr(mp.contiguous()), _MAP_DT[mp.dtype], _lib.ptr(srcs.contiguous()),
                                    _lib.ptr(dsts.contiguous()), N, H, W, D, *map(float, voxel_map), float(sigma),
                                    _lib.ptr(warped), _lib.ptr(ll), _lib.ptr(ws), ws.numel(), _lib.stream_ptr()))
    return ll


class TransformWrapper:
    """2D transforms of an nRows x nCols image domain (cpab/cpa2d/TransformWrapper.py:24-317),
    single level.  The domain is [0, nCols] x [0, nRows] in pixel units; dense
    points are the integer pixel coordinates (x_dense_img)."""

    def __init__(self, nRows: int, nCols: int, base=(4, 4), tess: str = "I", zero_v_across_bdry=(True, True),
                 scale_spatial: float = 1.0, scale_value: float = 100.0, nLevels: int = 1, device=None,
                 precision: torch.dtype = torch.float64, vol_preserve: bool = False, valid_outside=False):
        if nLevels != 1:
            raise NotImplementedError("multiscale registration is outside the built path (single level)")
        self.nRows, self.nCols = int(nRows), int(nCols)
        self.space = CpaSpace([0.0, 0.0], [float(nCols), float(nRows)], tuple(base), tess=tess,
                              zero_v_across_bdry=zero_v_across_bdry, device=device, precision=precision,
                              vol_preserve=vol_preserve, valid_outside=valid_outside)
        self.device = self.space.device
        self.scale_spatial, self.scale_value = scale_spatial, scale_value
        yy, xx = np.mgrid[0:self.nRows, 0:self.nCols]
        self.pts_src_dense = torch.as_tensor(np.stack([xx.ravel(), yy.ravel()], 1).astype(np.float64),
                                             device=self.device)
        p = default_params_flow_int(2)
        p["nStepsODEsolver"] = 10                  # TransformWrapper.py:126
        self.params_flow_int = p
        self.params_flow_int_coarse = dict(p, nTimeSteps=p["nTimeSteps"] // 10, dt=p["dt"] * 10)
        self.params_flow_int_fine = dict(p, nTimeSteps=p["nTimeSteps"] * 10, dt=p["dt"] / 10)

    def _params(self, int_quality: int) -> dict:
        return {0: self.params_flow_int, 1: self.params_flow_int_fine, -1: self.params_flow_int_coarse}[int_quality]

    def update_pat_from_theta(self, theta, level: int = 0):
        self.space.theta2Avees(theta)
        self.space.update_pat()

    def sample_from_the_prior(self, rng: np.random.Generator, length_scale: float | None = None):
        """theta ~ N(0, Sigma_CPA) with the wrapper's (scale_spatial, scale_value)."""
        from .space import Prior
        centers = self.space.geo.cells.mean(axis=1)
        d0 = np.linalg.norm(centers[0] - centers[1])
        ls = length_scale if length_scale is not None else self.scale_spatial * d0
        pr = Prior.create(self.space.geo, length_scale=ls, variance=self.scale_value ** 2)
        return pr.sample(1, rng)[0]

    def calc_T_fwd(self, pts_src, pts_fwd, level: int = 0, int_quality: int = 0):
        return self.space.calc_T_fwd(pts=pts_src, out=pts_fwd, **self._params(int_quality))

    def calc_T_inv(self, pts_src, pts_inv, level: int = 0, int_quality: int = 0):
        return self.space.calc_T_inv(pts=pts_src, out=pts_inv, **self._params(int_quality))

    def calc_v(self, level: int = 0, pts=None, v=None):
        return self.space.calc_v(pts=pts, out=v)

    def calc_trajectory(self, pts, mysign: int = 1, level: int = 0):
        return self.space.calc_trajectory(pts=pts, mysign=mysign, **self.params_flow_int)

    def calc_cell_idx(self, pts, cell_idx, level: int = 0):
        return self.space.calc_cell_idx(pts, cell_idx)

    def remap_fwd(self, pts_inv, img, img_wrapped_fwd):
        """img_wrapped_fwd = img o T (sample img at the T^-1 points), :261-270."""
        img_wrapped_fwd.zero_()
        return remap(pts_inv, img, out=img_wrapped_fwd)

    def remap_inv(self, pts_fwd, img, img_wrapped_inv):
        """img_wrapped_inv = img o T^-1 (sample img at the T points), :272-283."""
        img_wrapped_inv.zero_()
        return remap(pts_fwd, img, out=img_wrapped_inv)


class GaussianLogLikelihood:
    """ll(theta) = sum_i -0.5 (src(T_theta^-1(x_i)) - dst(x_i))^2 / sigma^2 over
    the pixel centres x_i of the unit square, for a batch of (theta, src, dst)."""

    def __init__(self, space: CpaSpace, src: torch.Tensor, dst: torch.Tensor, sigma_signal: float,
                 params_flow_int: dict | None = None, precision: torch.dtype | None = None):
        if space.dim != 2:
            raise ValueError("2D spaces only")
        self.space = space
        self.src = src if src.ndim == 3 else src.unsqueeze(0)
        self.dst = dst if dst.ndim == 3 else dst.unsqueeze(0)
        if self.src.shape != self.dst.shape or self.src.dtype != torch.float32:
            raise ValueError("src/dst must be float32 images of the same shape")
        self.src = self.src.contiguous()
        self.dst = self.dst.contiguous()
        self.N, self.H, self.W = self.src.shape
        self.nPts = self.H * self.W
        self.sign = -1        # the image is pulled back: calc_T_inv of the pixel grid
        self.sigma = float(sigma_signal)
        p = default_params_flow_int(2)
        if params_flow_int:
            p.update(params_flow_int)
        self.dt, self.nT, self.nODE = float(p["dt"]), int(p["nTimeSteps"]), int(p["nStepsODEsolver"])
        self.prec = _lib.CPAB_F64 if (precision or space.precision) == torch.float64 else _lib.CPAB_F32
        c = space._ctx
        self._ws = _ws(c.lib.cpab_register_workspace_bytes(c.h, self.N, self.H, self.W), space.device)
        self.nCalls = 0

    def batch(self, theta: torch.Tensor, warped: torch.Tensor | None = None,
              counters: torch.Tensor | None = None) -> torch.Tensor:
        """ll for theta [N, d] (N = number of image pairs), float64 [N]."""
        th = torch.as_tensor(theta, dtype=torch.float64, device=self.space.device).reshape(self.N, -1)
        sA, Tr = self.space.tables_from_theta(th, self.dt, -1)
        return self.batch_tables((sA, Tr), warped=warped, counters=counters)

    def batch_tables(self, tables, warped=None, counters=None, ll=None) -> torch.Tensor:
        sA, Tr = tables
        ll = torch.empty(self.N, dtype=torch.float64, device=self.space.device) if ll is None else ll
        c = self.space._ctx
        c.check(c.lib.cpab_register_ll(c.h, _lib.ptr(sA), _lib.ptr(Tr), self.N, _lib.ptr(self.src),
                                       _lib.ptr(self.dst), self.H, self.W, self.sigma, self.prec, self.dt, self.nT,
                                       self.nODE, _lib.ptr(ll), _lib.ptr(warped), _lib.ptr(self._ws),
                                       self._ws.numel(), _lib.ptr(counters), _lib.stream_ptr()))
        return ll

    def __call__(self, theta) -> float:
        """The reference's ll(theta) -> float (one image pair)."""
        if self.N != 1:
            raise ValueError("use batch() for several image pairs")
        self.nCalls += 1
        return float(self.batch(torch.as_tensor(theta).reshape(1, -1))[0].item())


class TransformWrapper3D:
    """3D transforms of an nRows x nCols x nSlices volume domain
    (cpab/cpa3d/TransformWrapper.py:21-289), single level.  The domain is
    [0, nCols] x [0, nRows] x [0, nSlices] in voxel units (XMAXS of :86-88);
    dense points are the integer voxel coordinates in the reference's order
    (np.mgrid[0:nRows, 0:nCols, 0:nSlices], z fastest), volumes are
    [nRows, nCols, nSlices]."""

    def __init__(self, nRows: int, nCols: int, nSlices: int, base=(2, 2, 2), tess: str = "II",
                 zero_v_across_bdry=(True, True, True), scale_spatial: float = 0.1, scale_value: float = 100.0,
                 nLevels: int = 1, device=None, precision: torch.dtype = torch.float64):
        if nLevels != 1:
            raise NotImplementedError("single level; see multiscale.py for the coarse-to-fine pyramid")
        if tess not in ("I", "II"):
            raise ValueError(tess, "tess must be in ['II','I']")
        self.nRows, self.nCols, self.nSlices = int(nRows), int(nCols), int(nSlices)
        self.space = CpaSpace([0.0, 0.0, 0.0], [float(nCols), float(nRows), float(nSlices)], tuple(base), tess=tess,
                              zero_v_across_bdry=zero_v_across_bdry, device=device, precision=precision)
        self.device = self.space.device
        self.scale_spatial, self.scale_value = scale_spatial, scale_value
        yy, xx, zz = np.mgrid[0:self.nRows, 0:self.nCols, 0:self.nSlices]
        self.pts_src_dense = torch.as_tensor(np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(np.float64),
                                             device=self.device)
        p = default_params_flow_int(3)
        p["nStepsODEsolver"] = 10                  # cpa3d/TransformWrapper.py:117
        self.params_flow_int = p
        self.params_flow_int_coarse = dict(p, nTimeSteps=p["nTimeSteps"] // 10, dt=p["dt"] * 10)
        self.params_flow_int_fine = dict(p, nTimeSteps=p["nTimeSteps"] * 10, dt=p["dt"] / 10)

    def _params(self, int_quality: int) -> dict:
        return {0: self.params_flow_int, 1: self.params_flow_int_fine, -1: self.params_flow_int_coarse}[int_quality]

    def update_pat_from_theta(self, theta, level: int = 0):
        self.space.theta2Avees(theta)
        self.space.update_pat()

    def calc_T_fwd(self, pts_src, pts_fwd, level: int = 0, int_quality: int = 0):
        return self.space.calc_T_fwd(pts=pts_src, out=pts_fwd, **self._params(int_quality))

    def calc_T_inv(self, pts_src, pts_inv, level: int = 0, int_quality: int = 0):
        return self.space.calc_T_inv(pts=pts_src, out=pts_inv, **self._params(int_quality))

    def calc_v(self, level: int = 0, pts=None, v=None):
        return self.space.calc_v(pts=pts, out=v)

    def calc_trajectory(self, pts, mysign: int = 1, level: int = 0):
        return self.space.calc_trajectory(pts=pts, mysign=mysign, **self.params_flow_int)

    def calc_cell_idx(self, pts, cell_idx, level: int = 0):
        return self.space.calc_cell_idx(pts, cell_idx)

    def remap_fwd(self, pts_inv, img, img_wrapped_fwd):
        """img_wrapped_fwd = img o T (sample img at the T^-1 points), :230-241."""
        img_wrapped_fwd.zero_()
        return remap3d(pts_inv, img, out=img_wrapped_fwd)

    def remap_inv(self, pts_fwd, img, img_wrapped_inv):
        """img_wrapped_inv = img o T^-1 (sample img at the T points), :243-253."""
        img_wrapped_inv.zero_()
        return remap3d(pts_fwd, img, out=img_wrapped_inv)


class GaussianLogLikelihood3D:
    """ll(theta) = sum_i -0.5 (src(T_theta^-1(x_i)) - dst(x_i))^2 / sigma^2 over
    the voxel centres x_i of the unit cube, for a batch of (theta, src, dst)
    volume triples [N, H, W, D] (one fused launch, cpab_register3d_ll)."""

    sign = -1             # the volume is pulled back: calc_T_inv of the voxel grid

    def __init__(self, space: CpaSpace, src: torch.Tensor, dst: torch.Tensor, sigma_signal: float,
                 params_flow_int: dict | None = None, precision: torch.dtype | None = None):
        if space.dim != 3:
            raise ValueError("3D spaces only")
        self.space = space
        self.src = (src if src.ndim == 4 else src.unsqueeze(0)).contiguous()
        self.dst = (dst if dst.ndim == 4 else dst.unsqueeze(0)).contiguous()
        if self.src.shape != self.dst.shape or self.src.dtype != torch.float32:
            raise ValueError("src/dst must be float32 volumes of the same shape")
        self.N, self.H, self.W, self.D = self.src.shape
        self.nPts = self.H * self.W * self.D
        self.sigma = float(sigma_signal)
        p = default_params_flow_int(3)
        if params_flow_int:
            p.update(params_flow_int)
        self.dt, self.nT, self.nODE = float(p["dt"]), int(p["nTimeSteps"]), int(p["nStepsODEsolver"])
        self.prec = _lib.CPAB_F64 if (precision or space.precision) == torch.float64 else _lib.CPAB_F32
        c = space._ctx
        self._ws = _ws(c.lib.cpab_register3d_workspace_bytes(c.h, self.N, self.H, self.W, self.D), space.device)
        self.nCalls = 0

    def batch(self, theta: torch.Tensor, warped: torch.Tensor | None = None,
              counters: torch.Tensor | None = None) -> torch.Tensor:
        th = torch.as_tensor(theta, dtype=torch.float64, device=self.space.device).reshape(self.N, -1)
        return self.batch_tables(self.space.tables_from_theta(th, self.dt, -1), warped=warped, counters=counters)

    def batch_tables(self, tables, warped=None, counters=None, ll=None) -> torch.Tensor:
        sA, Tr = tables
        ll = torch.empty(self.N, dtype=torch.float64, device=self.space.device) if ll is None else ll
        c = self.space._ctx
        c.check(c.lib.cpab_register3d_ll(c.h, _lib.ptr(sA), _lib.ptr(Tr), self.N, _lib.ptr(self.src),
                                         _lib.ptr(self.dst), self.H, self.W, self.D, self.sigma, self.prec, self.dt,
                                         self.nT, self.nODE, _lib.ptr(ll), _lib.ptr(warped), _lib.ptr(self._ws),
                                         self._ws.numel(), _lib.ptr(counters), _lib.stream_ptr()))
        return ll

    def __call__(self, theta) -> float:
        if self.N != 1:
            raise ValueError("use batch() for several volume pairs")
        self.nCalls += 1
        return float(self.batch(torch.as_tensor(theta).reshape(1, -1))[0].item())
