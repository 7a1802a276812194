"""CpaSpace: the reference's transform API on torch CUDA tensors.

Mirrors cpab/cpaNd/_CpaSpace.py (method names, argument order, the sign
convention of calc_T_fwd / calc_T_inv, the caller-allocated `out`, the
1D boundary clamp) with torch.Tensor in place of CpuGpuArray.  Every call
runs hand-written sm_100a kernels from libcpab_b200.so through the C ABI;
there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .space import TESS_I, TESS_II, Prior, SpaceGeometry, basis_from_reference_cache, build_space

_DT = {torch.float64: _lib.CPAB_F64, torch.float32: _lib.CPAB_F32}


def default_params_flow_int(dim: int) -> dict:
    """Defaults of cpab/cpa{1,2,3}d/calcs/_default_params_flow_int.py."""
    if dim == 1:
        return dict(dt=0.01, nTimeSteps=100, nStepsODEsolver=10)
    return dict(dt=0.0001, nTimeSteps=10, nStepsODEsolver=10)


class _Ctx:
    """Owns one cpab_ctx handle."""

    def __init__(self, geo: SpaceGeometry):
        lib = _lib.load()
        h = C.c_void_p()
        nCs = (C.c_int * 3)(*(list(geo.nCs) + [1] * (3 - geo.dim)))
        incs = (C.c_double * 3)(*(list(geo.incs) + [1.0] * (3 - geo.dim)))
        _lib.check(lib.cpab_ctx_create(C.byref(h), geo.dim, geo.tess_code, nCs, incs))
        self.h = h
        self.lib = lib

    def __del__(self):
        try:
            if self.h:
                self.lib.cpab_ctx_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def check(self, status: int) -> None:
        _lib.check(status, self.h)


class PAT:
    """Piecewise-affine transformation of one space: the per-cell matrices
    (Avees, device float64 [D]) plus cached signed matrices and exponentials
    (cpab/cpaNd/_PAT.py:48-59)."""

    def __init__(self, space: "CpaSpace", Avees: torch.Tensor | None = None):
        self.space = space
        self.nC = space.nC
        self.Avees = torch.zeros(space.D, dtype=torch.float64, device=space.device)
        self._cache: dict = {}
        if Avees is not None:
            self.update(Avees)

    def update(self, Avees) -> None:
        a = torch.as_tensor(Avees, dtype=torch.float64, device=self.space.device).reshape(-1)
        if a.numel() != self.space.D:
            raise ValueError(a.shape, self.space.D)
        self.Avees.copy_(a)
        self._cache.clear()

    @property
    def As(self) -> torch.Tensor:
        return self.Avees.view(self.nC, self.space.dim, self.space.dim + 1)

    def signed_tables(self, dt: float, sign: int, stream=None):
        key = (float(dt), int(sign))
        hit = self._cache.get(key)
        if hit is None:
            sA = torch.empty(self.space.D, dtype=torch.float64, device=self.space.device)
            Tr = torch.empty_like(sA)
            ctx = self.space._ctx
            ctx.check(ctx.lib.cpab_expm(ctx.h, _lib.ptr(self.Avees), 1, float(dt), int(sign),
                                        _lib.ptr(sA), _lib.ptr(Tr), _lib.stream_ptr(stream)))
            hit = (sA, Tr)
            self._cache[key] = hit
        return hit


class CpaSpace:
    """A CPA space over [XMINS, XMAXS] (XMINS must be 0, as in the reference,
    cpab/cpa2d/calcs/_CpaCalcs.py:38-39)."""

    def __init__(self, XMINS: Sequence[float], XMAXS: Sequence[float], nCs: Sequence[int],
                 zero_v_across_bdry: Sequence[bool] | None = None, vol_preserve: bool = False,
                 tess: str = TESS_II, valid_outside: bool | None = None, device=None,
                 precision: torch.dtype = torch.float64, reference_cache=None):
        """reference_cache: the reference's cache directory of subspaces
        (its <cache>/<dim>d/<subspace string>/subspace.pkl files); when it
        holds this space, its B is used (checked to span the same subspace),
        so theta values from the reference's runs map to the same A."""
        dim = len(nCs)
        if vol_preserve:
            raise NotImplementedError("volume-preserving spaces are outside the built path")
        if tess == TESS_I and dim == 2 and valid_outside:
            raise NotImplementedError("valid_outside=True is outside the built path")
        if any(float(x) != 0.0 for x in XMINS):
            raise ValueError("XMINS must be 0 (the cell lookup assumes it)")
        if precision not in _DT:
            raise TypeError(precision)
        self.dim = self.dim_domain = self.dim_range = dim
        self.tess = tess
        self.XMINS = np.asarray(XMINS, dtype=np.float64)
        self.XMAXS = np.asarray(XMAXS, dtype=np.float64)
        self.zero_v_across_bdry = tuple(zero_v_across_bdry if zero_v_across_bdry is not None else (True,) * dim)
        self.geo = build_space(dim, tuple(int(n) for n in nCs), tess, tuple(self.XMINS), tuple(self.XMAXS),
                               self.zero_v_across_bdry)
        if reference_cache is not None:
            B_ref = basis_from_reference_cache(self.geo, reference_cache)
            if B_ref is not None:
                self.geo = dataclasses.replace(self.geo, B=B_ref)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.precision = precision
        self.nCs = self.geo.nCs
        self.nC = self.geo.nC
        self.incs = self.geo.incs
        self.nHomoCoo = dim + 1
        self.lengthAvee = self.geo.lengthAvee
        self.Ashape = (dim, dim + 1)
        self.D = self.geo.D
        self.d = self.geo.d
        self.B_host = self.geo.B
        self.B = torch.as_tensor(np.ascontiguousarray(self.geo.B), device=self.device)
        self._ctx = _Ctx(self.geo)
        if dim == 1 and self.zero_v_across_bdry[0]:
            # threshold_krnl clamp of cpab/cpaNd/_CpaSpace.py:655-664
            self._ctx.check(self._ctx.lib.cpab_set_clamp(self._ctx.h, 1, float(self.XMINS[0]),
                                                         float(self.XMAXS[0])))
        self.pat = PAT(self)
        self.Avees = self.pat.Avees

    # ------------------------------------------------------------------ parameters
    def get_zeros_theta(self) -> np.ndarray:
        return np.zeros(self.d)

    def get_zeros_PA(self) -> np.ndarray:
        return np.zeros(self.D)

    def theta2Avees(self, theta, Avees=None):
        """A = B theta (cpab/cpaNd/_CpaSpace.py:366-376)."""
        th = torch.as_tensor(theta, dtype=torch.float64, device=self.device)
        res = self.B @ th
        if Avees is None:
            self.Avees.copy_(res)
            return self.Avees
        Avees.copy_(res) if isinstance(Avees, torch.Tensor) else np.copyto(Avees, res.cpu().numpy())
        return Avees

    def Avees2theta(self, Avees=None):
        a = self.Avees if Avees is None else torch.as_tensor(Avees, dtype=torch.float64, device=self.device)
        return self.B.T @ a

    def Avees2As(self, Avees=None):
        a = self.Avees if Avees is None else Avees
        return a.reshape(self.nC, *self.Ashape)

    def update_pat(self, Avees=None) -> None:
        self.pat.update(self.Avees if Avees is None else Avees)

    def create_prior(self, length_scale: float = 0.1, variance: float = 1.0, **kw) -> Prior:
        return Prior.create(self.geo, length_scale=length_scale, variance=variance, **kw)

    # ------------------------------------------------------------------ checks
    def _check_pts(self, pts: torch.Tensor, name: str = "pts") -> None:
        if not isinstance(pts, torch.Tensor):
            raise TypeError(type(pts))
        if pts.device.type != "cuda":
            raise ValueError(f"{name} must be a CUDA tensor")
        if pts.ndim != 2 or pts.shape[1] != self.dim:
            raise ValueError(f"{name}.shape = {tuple(pts.shape)}, expected (nPts, {self.dim})")
        if not pts.is_contiguous():
            raise ValueError(f"{name} must be C-contiguous")
        if pts.dtype not in _DT:
            raise ValueError(f"{name}.dtype = {pts.dtype}")

    def _flow(self, params: dict) -> tuple[float, int, int]:
        p = default_params_flow_int(self.dim)
        p.update(params)
        return float(p["dt"]), int(p["nTimeSteps"]), int(p["nStepsODEsolver"])

    # ------------------------------------------------------------------ transforms
    def calc_cell_idx(self, pts: torch.Tensor, cell_idx: torch.Tensor) -> torch.Tensor:
        """cpab/cpaNd/_CpaSpace.py:567 -> _CpaCalcs.calc_cell_idx (:59-88)."""
        self._check_pts(pts)
        if pts.dtype != torch.float64:
            raise ValueError(pts.dtype)
        if cell_idx.dtype != torch.int32 or cell_idx.numel() != pts.shape[0] or not cell_idx.is_contiguous():
            raise ValueError("cell_idx must be a contiguous int32 tensor with one entry per point")
        c = self._ctx
        c.check(c.lib.cpab_calc_cell_idx(c.h, _lib.ptr(pts), _lib.ptr(cell_idx), pts.shape[0], _lib.stream_ptr()))
        return cell_idx

    def calc_v(self, pat: PAT | None = None, pts: torch.Tensor | None = None, out: torch.Tensor | None = None,
               do_checks: bool = True) -> torch.Tensor:
        """v(x) = A_c [x; 1] (cpab/cpaNd/_CpaSpace.py:573-587)."""
        pat = pat or self.pat
        if pts is None:
            raise ValueError("Pts cannot be None")
        if out is None:
            raise ValueError("out Can't have None")
        self._check_pts(pts)
        self._check_pts(out, "out")
        if pts.dtype != torch.float64 or out.dtype != torch.float64 or out.shape != pts.shape:
            raise ValueError("calc_v works on float64 points with out.shape == pts.shape")
        c = self._ctx
        c.check(c.lib.cpab_calc_v(c.h, _lib.ptr(pat.Avees), _lib.ptr(pts), _lib.ptr(out), pts.shape[0],
                                  _lib.stream_ptr()))
        return out

    def _calc_T(self, pat, pts, mysign, out, scheme=_lib.SCHEME_REF, counters=None, **params_flow_int):
        pat = pat or self.pat
        if pts is None:
            raise ValueError
        if out is None:
            raise ValueError("You must pass the OUT argument")
        self._check_pts(pts)
        self._check_pts(out, "out")
        if out.dtype != pts.dtype or out.shape != pts.shape:
            raise ValueError("out must match pts in shape and dtype")
        if pts.data_ptr() == out.data_ptr():
            raise ValueError("pts and out cannot point to the same memory")
        dt, nT, nODE = self._flow(params_flow_int)
        sA, Tr = pat.signed_tables(dt, mysign)
        c = self._ctx
        c.check(c.lib.cpab_calc_T(c.h, _lib.ptr(sA), _lib.ptr(Tr), _lib.ptr(pts), _lib.ptr(out), pts.shape[0],
                                  _DT[pts.dtype], scheme, dt, nT, nODE, _lib.ptr(counters), _lib.stream_ptr()))
        return out

    def calc_T_fwd(self, pat=None, pts=None, do_checks=True, out=None, **params_flow_int):
        """T(x) (cpab/cpaNd/_CpaSpace.py:626-627)."""
        return self._calc_T(pat, pts, 1, out, **params_flow_int)

    def calc_T_inv(self, pat=None, pts=None, do_checks=True, out=None, **params_flow_int):
        """T^{-1}(x): the flow of -v (cpab/cpaNd/_CpaSpace.py:629-630)."""
        return self._calc_T(pat, pts, -1, out, **params_flow_int)

    def calc_T_simple(self, pat=None, pts=None, mysign=1, do_checks=True, out=None, **params_flow_int):
        """Midpoint-only integration (cpab/cpaNd/_CpaSpace.py:590-624)."""
        return self._calc_T(pat, pts, mysign, out, scheme=_lib.SCHEME_SIMPLE, **params_flow_int)

    def calc_T_exact(self, pat=None, pts=None, mysign=1, out=None, **params_flow_int):
        """The flow for time dt*nTimeSteps with cell-boundary hitting times:
        in 1D the closed form (cpab/cpa1d/calcs/ClosedFormInt.py:64-165); in
        2D/3D the reference's closed-form steps, with a step that leaves its
        cell re-integrated in nStepsODE sub-steps of the exact flow whose
        exits are resolved at the facet hitting times."""
        return self._calc_T(pat, pts, mysign, out, scheme=_lib.SCHEME_EXACT, **params_flow_int)

    def calc_trajectory(self, pat=None, pts=None, mysign=1, **params_flow_int) -> torch.Tensor:
        """[(1+nTimeSteps), nPts, dim] positions, row 0 = pts
        (cpab/cpaNd/_CpaSpace.py:688-703, _CpaCalcs.py:795-871)."""
        pat = pat or self.pat
        if pts is None:
            raise ValueError("pts cannot be None")
        self._check_pts(pts)
        if pts.dtype != torch.float64:
            raise ValueError(pts.dtype)
        dt, nT, nODE = self._flow(params_flow_int)
        sA, Tr = pat.signed_tables(dt, mysign)
        traj = torch.empty((nT + 1, pts.shape[0], self.dim), dtype=torch.float64, device=self.device)
        c = self._ctx
        c.check(c.lib.cpab_calc_trajectory(c.h, _lib.ptr(sA), _lib.ptr(Tr), _lib.ptr(pts), _lib.ptr(traj),
                                           pts.shape[0], dt, nT, nODE, _lib.stream_ptr()))
        return traj

    # ------------------------------------------------------------------ batches
    def tables_from_theta(self, theta: torch.Tensor, dt: float, mysign: int = 1, A_out: torch.Tensor | None = None,
                          out: tuple | None = None):
        """signed A and Trel for a batch theta [N, d] (one fused launch);
        written into out = (sA, Tr) ([N, D] float64 CUDA) when given."""
        th = theta.to(device=self.device, dtype=torch.float64).contiguous()
        if th.ndim != 2 or th.shape[1] != self.d:
            raise ValueError(th.shape)
        N = th.shape[0]
        if out is None:
            sA = torch.empty((N, self.D), dtype=torch.float64, device=self.device)
            Tr = torch.empty_like(sA)
        else:
            sA, Tr = out
            for t in (sA, Tr):
                if t.shape != (N, self.D) or t.dtype != torch.float64 or not t.is_contiguous() or \
                        t.device != self.device:
                    raise ValueError("out must be two contiguous float64 [N, D] tensors on the space's device")
        c = self._ctx
        c.check(c.lib.cpab_theta_to_trels(c.h, _lib.ptr(self.B), self.d, _lib.ptr(th), N, float(dt), int(mysign),
                                          _lib.ptr(A_out), _lib.ptr(sA), _lib.ptr(Tr), _lib.stream_ptr()))
        return sA, Tr

    def tables_from_A(self, A: torch.Tensor, dt: float, mysign: int = 1):
        """signed A and Trel for a batch of matrices A [N, D]."""
        A = A.to(device=self.device, dtype=torch.float64).contiguous()
        N = A.shape[0]
        sA = torch.empty((N, self.D), dtype=torch.float64, device=self.device)
        Tr = torch.empty_like(sA)
        c = self._ctx
        c.check(c.lib.cpab_expm(c.h, _lib.ptr(A), N, float(dt), int(mysign), _lib.ptr(sA), _lib.ptr(Tr),
                                _lib.stream_ptr()))
        return sA, Tr

    def calc_T_batched(self, tables, pts: torch.Tensor, out: torch.Tensor, offsets: torch.Tensor | None = None,
                       scheme: int = _lib.SCHEME_REF, counters: torch.Tensor | None = None,
                       workspace: torch.Tensor | None = None, **params_flow_int) -> torch.Tensor:
        """N transforms in one persistent launch.  tables = (signedA, Trels)
        [N, D] from tables_from_theta / tables_from_A with the same dt and sign.
        Points of instance i: pts[offsets[i]:offsets[i+1]] (offsets: CUDA
        int64 [N+1]) or, without offsets, N equal slices of pts."""
        sA, Tr = tables
        N = sA.shape[0]
        self._check_pts(pts)
        self._check_pts(out, "out")
        if out.dtype != pts.dtype or out.shape != pts.shape:
            raise ValueError("out must match pts")
        dt, nT, nODE = self._flow(params_flow_int)
        c = self._ctx
        if offsets is None:
            if pts.shape[0] % max(N, 1):
                raise ValueError("without offsets, nPts must be a multiple of N")
            n_uniform, ws, ws_bytes = pts.shape[0] // max(N, 1), None, 0
        else:
            if offsets.dtype != torch.int64 or offsets.numel() != N + 1 or offsets.device.type != "cuda":
                raise ValueError("offsets must be a CUDA int64 tensor of N+1 entries")
            n_uniform = 0
            ws_bytes = int(c.lib.cpab_batched_workspace_bytes(N))
            if workspace is None or workspace.numel() * workspace.element_size() < ws_bytes:
                workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
            ws = workspace
        c.check(c.lib.cpab_calc_T_batched(c.h, _lib.ptr(sA), _lib.ptr(Tr), _lib.ptr(pts), _lib.ptr(out), N,
                                          _lib.ptr(offsets), n_uniform, _lib.ptr(ws), ws_bytes, _DT[pts.dtype],
                                          scheme, dt, nT, nODE, _lib.ptr(counters), _lib.stream_ptr()))
        return out

    def capture_batched(self, n_theta: int, pts: torch.Tensor, out: torch.Tensor,
                        offsets: torch.Tensor | None = None, mysign: int = 1, scheme: int = _lib.SCHEME_REF,
                        counters: torch.Tensor | None = None, **params_flow_int) -> "BatchedStep":
        """One batched step -- theta [n_theta, d] -> A = B theta -> expm ->
        integration of every instance's points -- captured in a CUDA graph
        (replaces the reference's per-call launch path, cpab/gpu/Calcs.py:454-624,
        for a batch whose shapes repeat).  pts, out, offsets and counters are
        the graph's fixed buffers: refill them in place between replays."""
        return BatchedStep(self, n_theta, pts, out, offsets, mysign, scheme, counters, **params_flow_int)

    def calc_T_batched_host(self, theta, pts_host: torch.Tensor, out_host: torch.Tensor, offsets_host,
                            mysign: int = 1, scheme: int = _lib.SCHEME_REF, chunks: int = 16,
                            **params_flow_int) -> torch.cuda.Event:
        """calc_T_batched for inputs and outputs in (pinned) HOST memory.

        The batch is cut into `chunks` contiguous groups of instances; group
        k+1 is copied in while group k is integrated and group k-1 is copied
        out (three streams, three device buffers).  The first two and last two
        groups carry 1/4 and 1/2 of an inner group's points, so the copy-in
        before the first integration and the copy-out after the last one --
        the stretches where the host link carries one direction only -- are
        short.  The device buffers belong to the space and are reused by the
        next call once their previous contents are copied out (events); every
        tensor used on a side stream is recorded on it, so freeing or growing
        a buffer never hands memory in use to another allocation.
        theta: [N, d] (host or device); offsets_host: int64 [N+1] (host).
        Returns an event recorded on the current stream once out_host is
        complete; the current stream waits for it."""
        dt, nT, nODE = self._flow(params_flow_int)
        offs = np.asarray(offsets_host, dtype=np.int64)
        N = offs.size - 1
        dev = self.device
        cur = torch.cuda.current_stream(dev)
        if not hasattr(self, "_pipe_streams"):
            self._pipe_streams = [torch.cuda.Stream(device=dev) for _ in range(3)]
            self._pipe_pool = []
        s_in, s_cmp, s_out = self._pipe_streams
        th = torch.as_tensor(theta, dtype=torch.float64)
        th = th.pin_memory().to(dev, non_blocking=True) if th.device.type == "cpu" else th.to(dev)
        tables = self.tables_from_theta(th, dt, mysign)
        for t in tables:
            t.record_stream(s_cmp)
        ev_tables = torch.cuda.Event()
        ev_tables.record(cur)
        total = int(offs[-1])
        chunks = max(1, min(int(chunks), N))
        groups = _pipeline_groups(offs, chunks)
        maxpts = max(int(offs[b] - offs[a]) for a, b in groups)
        dim = self.dim
        dt_ = pts_host.dtype
        nbuf = min(3, len(groups))
        ws_need = int(self._ctx.lib.cpab_batched_workspace_bytes(N)) + 256
        pool = self._pipe_pool
        for i in range(nbuf):
            buf = pool[i] if i < len(pool) else None
            if buf is None or buf["x"].dtype != dt_ or buf["x"].shape[0] < maxpts or buf["x"].shape[1] != dim or \
                    buf["off"].numel() < len(offs) or buf["ws"].numel() < ws_need:
                # the old buffers were recorded on the streams that used them: freeing is safe
                buf = dict(x=torch.empty((maxpts, dim), dtype=dt_, device=dev),
                           o=torch.empty((maxpts, dim), dtype=dt_, device=dev),
                           off=torch.empty(len(offs), dtype=torch.int64, device=dev),
                           ws=torch.empty(ws_need, dtype=torch.uint8, device=dev),
                           ev_free=buf["ev_free"] if buf is not None else None)
                if i < len(pool):
                    pool[i] = buf
                else:
                    pool.append(buf)
        off_pin = torch.empty((len(groups), len(offs)), dtype=torch.int64).pin_memory()
        ev_last = None
        for k, (a, b) in enumerate(groups):
            buf = pool[k % nbuf]
            o0, o1 = int(offs[a]), int(offs[b])
            n = o1 - o0
            off_pin[k, :b - a + 1] = torch.from_numpy(offs[a:b + 1] - o0)
            if buf["ev_free"] is not None:          # its previous group (this call or the last) is copied out
                s_in.wait_event(buf["ev_free"])
            with torch.cuda.stream(s_in):
                buf["x"][:n].copy_(pts_host[o0:o1], non_blocking=True)
                buf["off"][:b - a + 1].copy_(off_pin[k, :b - a + 1], non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(s_in)
            s_cmp.wait_event(ev_in)
            s_cmp.wait_event(ev_tables)
            with torch.cuda.stream(s_cmp):
                self.calc_T_batched((tables[0][a:b], tables[1][a:b]), buf["x"][:n], buf["o"][:n],
                                    offsets=buf["off"][:b - a + 1], scheme=scheme, workspace=buf["ws"], **params_flow_int)
                ev_c = torch.cuda.Event()
                ev_c.record(s_cmp)
            s_out.wait_event(ev_c)
            with torch.cuda.stream(s_out):
                out_host[o0:o1].copy_(buf["o"][:n], non_blocking=True)
                ev_o = torch.cuda.Event()
                ev_o.record(s_out)
            for key, st in (("x", s_in), ("off", s_in), ("x", s_cmp), ("o", s_cmp), ("off", s_cmp), ("ws", s_cmp),
                            ("o", s_out)):
                buf[key].record_stream(st)
            buf["ev_free"] = ev_o
            ev_last = ev_o
        cur.wait_event(ev_last)
        done = torch.cuda.Event()
        done.record(cur)
        return done

    def cancel(self) -> None:
        """Stop running and future launches of this space between tiles (see cpab_cancel)."""
        c = self._ctx
        c.check(c.lib.cpab_cancel(c.h))

    def clear_cancel(self) -> None:
        c = self._ctx
        c.check(c.lib.cpab_clear_cancel(c.h))

    def set_launch(self, block: int = 0, ctas_per_sm: int = 0, tile_pts: int = 0, cell_sort: bool | None = None,
                   max_ctas: int | None = None) -> None:
        c = self._ctx
        c.check(c.lib.cpab_set_launch(c.h, block, ctas_per_sm, tile_pts))
        if cell_sort is not None:
            c.check(c.lib.cpab_set_cell_sort(c.h, int(bool(cell_sort))))
        if max_ctas is not None:
            c.check(c.lib.cpab_set_max_ctas(c.h, int(max_ctas)))

    def __repr__(self) -> str:
        return self.geo.subspace_string


def _pipeline_groups(offs: np.ndarray, chunks: int) -> list[tuple[int, int]]:
    """Contiguous instance groups [a, b) for the host-buffer pipeline: point
    counts in the proportions 1/4, 1/2, 1, ..., 1, 1/2, 1/4 (equal when there
    are fewer than six groups), cut at instance boundaries; empty groups are
    dropped."""
    N = offs.size - 1
    total = int(offs[-1])
    w = np.ones(chunks)
    if chunks >= 6:
        w[[0, -1]] = 0.25
        w[[1, -2]] = 0.5
    frac = np.cumsum(w)[:-1] / w.sum()
    cuts = np.searchsorted(offs, frac * total)
    bounds = np.unique(np.concatenate([[0], cuts, [N]]))
    return [(int(a), int(b)) for a, b in zip(bounds[:-1], bounds[1:]) if b > a]


class BatchedStep:
    """A batched transform step replayed from a CUDA graph.

    The graph holds the three launches of a step -- the fused
    theta -> A -> expm prologue, the ragged batch's tile prefix and the
    persistent integration kernel -- on fixed buffers: `theta` (owned here,
    [n_theta, d] float64), the caller's `pts`, `out`, `offsets` and
    `counters`, and an owned workspace and table pair.  Construction runs the
    step once eagerly (kernel attributes, launch shapes) and captures it on a
    side stream; `__call__` replays it on the current stream.  The launch
    shape (CpaSpace.set_launch / the autotuner) is fixed at capture."""

    def __init__(self, space: CpaSpace, n_theta: int, pts: torch.Tensor, out: torch.Tensor,
                 offsets: torch.Tensor | None, mysign: int, scheme: int, counters: torch.Tensor | None,
                 **params_flow_int):
        self.space = space
        dev = space.device
        self.dt, self.nT, self.nODE = space._flow(params_flow_int)
        self.params = dict(dt=self.dt, nTimeSteps=self.nT, nStepsODEsolver=self.nODE)
        self.mysign, self.scheme = int(mysign), int(scheme)
        self.pts, self.out, self.offsets, self.counters = pts, out, offsets, counters
        self.theta = torch.zeros((n_theta, space.d), dtype=torch.float64, device=dev)
        self.tables = (torch.empty((n_theta, space.D), dtype=torch.float64, device=dev),
                       torch.empty((n_theta, space.D), dtype=torch.float64, device=dev))
        ws_bytes = int(space._ctx.lib.cpab_batched_workspace_bytes(n_theta)) if offsets is not None else 0
        self.workspace = torch.empty(max(ws_bytes, 256), dtype=torch.uint8, device=dev)
        self._launches()                      # eager: sets kernel attributes before capture
        torch.cuda.current_stream(dev).synchronize()
        self.graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            self.graph.capture_begin(capture_error_mode="thread_local")
            try:
                self._launches()
            finally:
                self.graph.capture_end()
        torch.cuda.current_stream(dev).wait_stream(side)

    def _launches(self) -> None:
        sp = self.space
        sp.tables_from_theta(self.theta, self.dt, self.mysign, out=self.tables)
        sp.calc_T_batched(self.tables, self.pts, self.out, offsets=self.offsets, scheme=self.scheme,
                          counters=self.counters, workspace=self.workspace, **self.params)

    def __call__(self, theta: torch.Tensor | None = None) -> torch.Tensor:
        """Replay the step (after copying `theta` into the graph's buffer when
        given); returns `out`."""
        if theta is not None:
            self.theta.copy_(torch.as_tensor(theta, dtype=torch.float64), non_blocking=True)
        self.graph.replay()
        return self.out
