"""Autotuner for the integration launch shape.

Candidates: threads per CTA, points per CTA tile, cell-sort on/off.  Each is
timed with CUDA events on a sample of the caller's batch (its first whole
instances, up to `sample_points` points), the fastest kept, and the choice cached per
(GPU name, dim, tessellation, cell count, precision, scheme) in memory and in
a JSON file (CPAB_B200_CACHE directory).  Results never depend on the choice:
every configuration runs each point through the same arithmetic.
"""
from __future__ import annotations

import itertools
import json
import os
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .cpa_space import CpaSpace

CANDIDATES = dict(block=(128, 256), tile_pts=(1024, 2048, 4096), cell_sort=(False, True))
_memo: dict = {}


def _cache_file() -> Path | None:
    d = os.environ.get("CPAB_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cpabdiffeo_b200"))
    if d in ("", "0", "off"):
        return None
    return Path(d) / "autotune.json"


def _key(space: CpaSpace, scheme: int) -> str:
    name = torch.cuda.get_device_name(space.device)
    prec = "f64" if space.precision == torch.float64 else "f32"
    return f"{name}|{space.dim}|{space.tess}|{space.nC}|{prec}|{scheme}"


def _load() -> dict:
    f = _cache_file()
    if f is None or not f.exists():
        return {}
    try:
        return json.loads(f.read_text())
    except (OSError, ValueError):
        return {}


def _store(key: str, cfg: dict) -> None:
    f = _cache_file()
    if f is None:
        return
    try:
        f.parent.mkdir(parents=True, exist_ok=True)
        data = _load()
        data[key] = cfg
        tmp = f.with_suffix(f".{os.getpid()}.tmp")
        tmp.write_text(json.dumps(data, indent=1))
        os.replace(tmp, f)
    except OSError:
        pass


def apply(space: CpaSpace, cfg: dict) -> None:
    space.set_launch(block=int(cfg["block"]), tile_pts=int(cfg["tile_pts"]), cell_sort=bool(cfg["cell_sort"]))


def sample_extent(n_inst_total: int, n_pts_total: int, offsets, sample_points: int) -> tuple[int, int]:
    """(instances, points) of the tuning sample: the batch's first whole
    instances with their own points.  Ragged (offsets: host int64 [N+1]): the
    instances up to the one whose points reach `sample_points`, and the next
    one; N equal slices (offsets None): as many whole instances as fit in
    `sample_points`.  At least one instance either way."""
    if offsets is not None:
        n_inst = int(np.searchsorted(offsets, sample_points)) + 1
        n_inst = max(1, min(n_inst, len(offsets) - 1))
        return n_inst, int(offsets[n_inst])
    n_per = n_pts_total // max(1, n_inst_total)
    n_inst = max(1, min(n_inst_total, sample_points // max(1, n_per)))
    return n_inst, n_inst * n_per


def tune(space: CpaSpace, tables, pts: torch.Tensor, offsets: torch.Tensor | None, scheme: int,
         sample_points: int = 4_000_000, reps: int = 3, use_cache: bool = True, **params_flow_int) -> dict:
    """Pick and apply the fastest launch shape for this batch; returns it (with its time)."""
    key = _key(space, scheme)
    if use_cache:
        hit = _memo.get(key) or _load().get(key)
        if hit:
            _memo[key] = hit
            apply(space, hit)
            return hit
    sA, Tr = tables
    offs = offsets.cpu().numpy() if offsets is not None else None
    n_inst, n_pts = sample_extent(sA.shape[0], pts.shape[0], offs, sample_points)
    sub_tables, x = (sA[:n_inst], Tr[:n_inst]), pts[:n_pts]
    sub_off = offsets[:n_inst + 1] if offsets is not None else None
    out = torch.empty_like(x)
    cand = [dict(block=b, tile_pts=t, cell_sort=s) for b, t, s in
            itertools.product(CANDIDATES["block"], CANDIDATES["tile_pts"], CANDIDATES["cell_sort"])]
    best, best_ms = None, float("inf")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for c in cand:
        apply(space, c)
        space.calc_T_batched(sub_tables, x, out, offsets=sub_off, scheme=scheme, **params_flow_int)   # warm
        ev0.record()
        for _ in range(reps):
            space.calc_T_batched(sub_tables, x, out, offsets=sub_off, scheme=scheme, **params_flow_int)
        ev1.record()
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1) / reps
        if ms < best_ms:
            best, best_ms = c, ms
    best = dict(best, ms_sample=best_ms, sample_points=int(x.shape[0]))
    apply(space, best)
    _memo[key] = best
    if use_cache:
        _store(key, best)
    return best
