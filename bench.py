"""Benchmark of the batched CPAB transform (one JSON line on stdout).

Workload (the batched 1D configuration): [0,1] split into nC=100 equal
cells, zero-velocity boundary; 4096 theta from the Gaussian prior (length
scale 0.1, variance 1); instance i transforms its own n_i = floor(10^U(3,5))
uniform points (~8.8e7 in total), FP32 points; integration time 1.0.  The
timed step integrates in closed form across cell boundaries (hitting times
in FP64, cpab/cpa1d/calcs/ClosedFormInt.py restated on the GPU): one fused
prologue launch (theta -> A -> expm for all 4096) and one persistent
integration launch.  Each run checks the result against the reference's own
calc_T scheme in FP64 (dt=0.02 x 50 steps, nStepsODE=100) on a sample of
instances and reports the error (must stay <= 1e-5); the same workload
through the REF scheme on the GPU is reported beside it.  Seeded synthetic
data (seed 1).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value`  : points/s over all ranks with inputs resident in HBM (device time,
           max over ranks); the inputs (352 MB of points) exceed L2.
`e2e`    : the same through CpaSpace.calc_T_batched with pinned host buffers,
           the H2D copy of theta/offsets/points and the D2H copy of the
           transformed points inside the timed region.
--impl reference: the reference's own kernel sources compiled for the host
           (oracle/_ref) in FP64 with all host threads on a bounded sample per
           step; with N > 1 only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "CPAB points/sec batched+served vs plain per-call at <=1e-5 err; p50/p99 latency"
UNIT = "points/s"
N_THETA, NC, SEED = 4096, 100, 1
DT, NT, NODE = 0.02, 50, 100
WORKLOAD = "batched_1d_nc100_4096theta_ragged_1e3_1e5"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the cpu baseline and the 2D plain-vs-batched leg")
    ap.add_argument("--theta", type=int, default=N_THETA)
    ap.add_argument("--e2e-chunks", type=int, default=16,
                    help="instance groups of the host-buffer pipeline (copy in / integrate / copy out overlap)")
    ap.add_argument("--serve-seconds", type=float, default=2.0,
                    help="seconds of Poisson arrivals at 2000 req/s for the serving leg; 0 skips serving")
    ap.add_argument("--serve-sustained-seconds", type=float, default=10.0,
                    help="seconds of arrivals at 80%% of the measured serving capacity; 0 skips that run")
    ap.add_argument("--workload", default="batched_1d",
                    choices=["batched_1d", "batched_2d_nc64", "exact_2d_nc64", "remap_ssd", "mcmc_c3", "serving"],
                    help="batched_1d: the headline (1D nC=100, 4096 theta, ragged); batched_2d_nc64: the reference "
                         "scheme in FP32 on 2D tess I 4x4 (nC=64), 4096 theta x 8192 points, for the "
                         "integration kernel's FP32 roofline; exact_2d_nc64: the same through the exact scheme "
                         "(facet hitting times); remap_ssd: remap + SSD of 256 pairs of 256x256 "
                         "images through FP32 maps, for its HBM roofline; mcmc_c3: 256-chain MCMC registration of "
                         "256x256 FP32 image pairs, for the fused likelihood kernel's roofline; serving: only the "
                         "serving legs (capacity, 200 req/s, sustained, 2000 req/s), one JSON line")
    return ap.parse_args()


def make_workload(rank: int, n_theta: int):
    from cpabdiffeo_b200.space import Prior, build_space
    geo = build_space(1, (NC,), "II")
    prior = Prior.create(geo, length_scale=0.1, variance=1.0)
    rng = np.random.default_rng(SEED + 1000 * rank)
    theta = prior.sample(n_theta, rng)
    sizes = np.floor(10 ** rng.uniform(3, 5, size=n_theta)).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    pts = rng.uniform(0, 1, size=(int(offsets[-1]), 1)).astype(np.float32)
    return geo, theta, sizes, offsets, pts


class ClockSampler:
    """SM clocks, power and clock-event reasons sampled while the timed region
    runs: NVML every 10 ms on a host thread (nvidia-smi -lms 200 when NVML is
    unavailable).  The sampler has taken its first sample before __enter__
    returns and takes a last one on __exit__, so even a short timed region is
    covered."""

    # NVML clock-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples: list[tuple] = []   # (sm_mhz, sm_max_mhz, power_w, set of reasons)
        self.stop = threading.Event()
        self.t = None
        self.proc = None
        self.source = None

    def _bus_id(self) -> str | None:
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            return f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        except Exception:
            return None

    def _nvml_loop(self, nv, h, first: threading.Event):
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while True:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(smax), pw,
                                     {k for k, b in self.REASONS.items() if bits & b}))
            except Exception:
                pass
            first.set()
            if self.stop.wait(0.01):
                break

    def _smi_loop(self, first: threading.Event):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                try:
                    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                    self.samples.append((float(f[1]), float(f[2]), float(f[3]),
                                         {nm for nm, v in zip(names, f[5:9]) if v.lower() == "active"}))
                except ValueError:
                    pass
            first.set()

    def __enter__(self):
        first = threading.Event()
        bus = self._bus_id()
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByPciBusId(bus) if bus else nv.nvmlDeviceGetHandleByIndex(self.index)
            self.nv = nv
            self.t = threading.Thread(target=self._nvml_loop, args=(nv, h, first), daemon=True)
            self.source = "nvml 10 ms"
        except Exception:
            try:
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={bus or self.index}", f"--query-gpu={self.FIELDS}",
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.t = threading.Thread(target=self._smi_loop, args=(first,), daemon=True)
                self.source = "nvidia-smi 200 ms"
            except OSError:
                return self
        self.t.start()
        first.wait(10.0)
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.proc is not None:
            time.sleep(0.25)               # one more nvidia-smi line after the timed region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.t is not None:
            self.t.join(timeout=5)

    def summary(self) -> dict:
        sm = [s[0] for s in self.samples]
        reasons = set().union(*[s[3] for s in self.samples]) if self.samples else set()
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": self.samples[-1][1] if self.samples else None,
                "sm_mhz_min": min(sm) if sm else None,
                "power_w_max": max(s[2] for s in self.samples) if self.samples else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": self.source}


_PEAKS: dict = {}


def measured_peaks(torch) -> dict:
    """FP32 / FP64 SIMT throughput measured here (cuBLAS SGEMM with TF32 off,
    DGEMM): the denominators for the integration kernel, which runs on the
    FP32 / FP64 pipes.  HBM from MEASURED_PEAKS.json."""
    if _PEAKS:
        return _PEAKS
    out = _PEAKS
    try:
        out.update(json.loads((ROOT / "MEASURED_PEAKS.json").read_text()))
    except (OSError, ValueError):
        out["hbm_gbs"] = 6650.0
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    for name, dt, n in (("fp32_simt_tflops", torch.float32, 8192), ("fp64_tflops", torch.float64, 4096)):
        a = torch.randn(n, n, device="cuda", dtype=dt)
        b = torch.randn(n, n, device="cuda", dtype=dt)
        for _ in range(2):
            a @ b
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = 1e30
        for _ in range(5):
            s.record()
            a @ b
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e))
        out[name] = 2 * n ** 3 / (best * 1e-3) / 1e12
        del a, b
    torch.backends.cuda.matmul.allow_tf32 = prev
    return out


# DRAM bytes per launch measured with ncu (dram__bytes_read.sum +
# dram__bytes_write.sum, one captured launch of the timed region):
#  * k_exact1d on the 2048-theta case (42.7 M points): 303.4 MB, 7.10 B/point,
#    scaled to a launch by the points it processes;
#  * k_integrate on the 2D 4096 x 8192-point workload: 587.9 MB per launch;
#  * k_remap_ssd_bulk on 256 pairs of 256^2 images: 273.0 MB per launch.
TRAFFIC_EXACT1D_BYTES_PER_POINT = 303.38e6 / 42737756
# Pipe utilisation of k_exact1d from the same capture (ncu, % of each pipe's
# peak over the active cycles; FMA-heavy over the elapsed cycles).
PIPES_EXACT1D = {"fp64_pct": 22.0, "fp32_fma_pct": 18.2, "fp32_fma_heavy_pct_elapsed": 30.5, "alu_pct": 31.5,
                 "issue_active_pct": 73.1, "source": "ncu --set full, one launch of the 2048-theta case"}
TRAFFIC_2D_BYTES_PER_LAUNCH = 587.94e6
TRAFFIC_REMAP_BYTES_PER_LAUNCH = 272.95e6

# Closed-form segment cost model (FP64 operations): per cell visit the
# crossing test and hitting time take 10 arithmetic operations plus one log,
# the final in-cell evaluation 6 plus one exp; log and exp are counted as 20
# operations each (range reduction + a degree ~8 polynomial).
EXACT_FLOP_PER_VISIT = 30
EXACT_FLOP_PER_POINT = 26


def flops_exact(cnt) -> float:
    return float(cnt[0] * EXACT_FLOP_PER_VISIT + cnt[3] * EXACT_FLOP_PER_POINT)


def flops_from_counters(cnt, dim=1) -> float:
    """Algorithmic FP ops of the REF scheme from device counters:
    per closed-form attempt 2*C_cell + M, per midpoint sub-step C_cell + 2M + 4D,
    with M = 2 D^2 (affine apply) and C_cell = 5 (1D box lookup)."""
    C_cell = {1: 5, 2: 24, 3: 36}[dim]
    M = 2 * dim * dim
    attempts = cnt[0] + cnt[1]
    return float(attempts * (2 * C_cell + M) + cnt[2] * (C_cell + 2 * M + 4 * dim))


def cpu_reference_rate(theta, offsets, pts, geo, budget_pts: int, rank_seed: int = 0):
    """The reference's calc_T (host-compiled, FP64, all threads) on the first
    instances covering ~budget_pts points.  Returns (points/s, sample text, kind, cores)."""
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    n_inst = int(np.searchsorted(offsets, budget_pts)) + 1
    n_inst = max(1, min(n_inst, len(offsets) - 1))
    t0 = time.perf_counter()
    npts = 0
    for i in range(n_inst):
        A = (geo.B @ theta[i]).reshape(NC, 2)
        sA, Tr = O.expm_cells(1, A, DT, 1)
        x = pts[offsets[i]:offsets[i + 1]].astype(np.float64)
        if kind == "reference":
            out = O.ref_calc_T(1, 2, geo.nCs, geo.incs, Tr, sA, x, DT, NT, NODE, geo.nC)
        else:
            out, _ = O.calc_T(O.tess_struct(1, 2, geo.nCs, geo.incs), Tr, sA, x, DT, NT, NODE)
        O.clamp_1d(out)
        npts += x.shape[0]
    dt = time.perf_counter() - t0
    return npts / dt, f"first {n_inst} of {len(offsets) - 1} instances ({npts} points), FP64", kind, O.nproc(), dt


def cpu_closed_form_rate(theta, offsets, pts, geo, budget_pts: int):
    """The closed form (the oracle's C restatement of ClosedFormInt, FP64,
    OpenMP over points, all host threads) on the first instances covering
    ~budget_pts points.  Returns (points/s, sample text, cores)."""
    from oracle import oracle as O
    n_inst = int(np.searchsorted(offsets, budget_pts)) + 1
    n_inst = max(1, min(n_inst, len(offsets) - 1))
    As = [(geo.B @ theta[i]).reshape(NC, 2) for i in range(n_inst)]
    xs = [pts[offsets[i]:offsets[i + 1]].astype(np.float64)[:, 0] for i in range(n_inst)]
    O.closed_form_1d(As[0], NC, xs[0], DT * NT)          # warm the library and the threads
    t0 = time.perf_counter()
    npts = 0
    for A, x in zip(As, xs):
        O.closed_form_1d(A, NC, x, DT * NT)
        npts += x.size
    dt = time.perf_counter() - t0
    return npts / dt, f"first {n_inst} of {len(offsets) - 1} instances ({npts} points), FP64", O.nproc()


def run_reference(args, rank, world):
    if rank != 0:
        return
    geo, theta, sizes, offsets, pts = make_workload(0, args.theta)
    budget = 150_000
    for _ in range(args.warmup):
        cpu_reference_rate(theta, offsets, pts, geo, budget)
    rates, secs, sample, kind, cores = [], 0.0, "", "", 1
    for _ in range(args.steps):
        r, sample, kind, cores, dt = cpu_reference_rate(theta, offsets, pts, geo, budget)
        rates.append(r)
        secs += dt
    value = float(np.mean(rates))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded prior draws, uniform points)",
            "config": {"workload": WORKLOAD, "scheme": "ref calc_T dt=0.02 nT=50 nODE=100", "sample": sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def plain_vs_batched_2d(torch, dev):
    """North-star comparison on the 2D nC=64 workload: FP32 batched (one launch
    for all theta) vs the plain path (one theta per call: host A = B theta,
    expm launch, calc_T launch, stream sync), 4096 points per theta."""
    from cpabdiffeo_b200 import _lib
    from cpabdiffeo_b200.cpa_space import CpaSpace
    from cpabdiffeo_b200.space import Prior
    sp64 = CpaSpace([0, 0], [1, 1], (4, 4), tess="I", device=dev, precision=torch.float64)
    sp32 = CpaSpace([0, 0], [1, 1], (4, 4), tess="I", device=dev, precision=torch.float32)
    rng = np.random.default_rng(0)
    nth, npt = 1024, 4096
    theta = Prior.create(sp64.geo, 0.1, 1.0).sample(nth, rng)
    x = rng.uniform(0, 1, size=(nth * npt, 2))
    p = dict(dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    # plain: first 64 theta, one call each (host A = B theta, expm launch, calc_T launch, stream sync),
    # in FP64 (the drop-in default) and in FP32 (the batched arm's precision)
    n_plain = 64

    def plain_rate(sp, dtype):
        xs = torch.as_tensor(x[:npt], device=dev, dtype=dtype)
        out = torch.empty_like(xs)
        for rep in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for i in range(n_plain):
                sp.update_pat(sp.B_host @ theta[i])
                sp.calc_T_fwd(pts=xs, out=out, **p)
                torch.cuda.current_stream().synchronize()
            t_plain = time.perf_counter() - t0
        return n_plain * npt / t_plain

    plain = plain_rate(sp64, torch.float64)
    plain32 = plain_rate(sp32, torch.float32)
    xb = torch.as_tensor(x, device=dev, dtype=torch.float32)
    ob = torch.empty_like(xb)
    th = torch.as_tensor(theta, device=dev)

    from cpabdiffeo_b200 import autotune
    autotune.tune(sp32, sp32.tables_from_theta(th, DT, 1), xb, None, _lib.SCHEME_REF, sample_points=1 << 20, **p)

    def step():
        tables = sp32.tables_from_theta(th, DT, 1)
        sp32.calc_T_batched(tables, xb, ob, **p)

    for _ in range(3):
        step()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(5):
        step()
    e.record()
    e.synchronize()
    batched = 5 * nth * npt / (s.elapsed_time(e) * 1e-3)
    return {"workload": "2d_tessI_4x4_nc64_1024theta_x_4096pts", "batched_points_per_s": batched,
            "batched_precision": "f32", "plain_per_call_f32_points_per_s": plain32,
            "plain_per_call_f64_points_per_s": plain, "ratio": batched / plain32,
            "ratio_precision": "f32 batched / f32 plain (same scheme, same precision)",
            "ratio_vs_f64_plain": batched / plain}


def other_configs(torch, dev) -> dict:
    """Bounded measurements of the other configurations (device-timed, CUDA events)."""
    from scipy.ndimage import gaussian_filter

    from cpabdiffeo_b200.autograd import transform
    from cpabdiffeo_b200.cpa_space import CpaSpace
    from cpabdiffeo_b200.mcmc import BatchedMetropolis
    from cpabdiffeo_b200.registration import GaussianLogLikelihood, remap
    from cpabdiffeo_b200.space import Prior, pixel_centers
    out = {}
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    p = dict(dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)

    # 2D nC=64, single theta, FP64: 512x512 pixel centres forward and inverse, remap of a 512^2 image
    sp = CpaSpace([0, 0], [1, 1], (4, 4), tess="I", device=dev)
    rng = np.random.default_rng(0)
    th = Prior.create(sp.geo, 0.1, 1.0).sample(1, rng)[0]
    sp.update_pat(sp.B @ torch.as_tensor(th, device=dev))
    x = torch.as_tensor(pixel_centers(512, 512), device=dev)
    y, z = torch.empty_like(x), torch.empty_like(x)
    img = torch.as_tensor(gaussian_filter(rng.uniform(0, 1, (512, 512)).astype(np.float32), 8.0), device=dev)
    warped = torch.empty_like(img)
    for _ in range(3):
        sp.calc_T_fwd(pts=x, out=y, **p)
        sp.calc_T_inv(pts=x, out=z, **p)
        remap(z, img, out=warped, pixel_map=(512, -0.5, 512, -0.5))
    a, b, c, d = ev(), ev(), ev(), ev()
    a.record()
    for _ in range(5):
        sp.calc_T_fwd(pts=x, out=y, **p)
    b.record()
    for _ in range(5):
        sp.calc_T_inv(pts=x, out=z, **p)
    c.record()
    for _ in range(5):
        remap(z, img, out=warped, pixel_map=(512, -0.5, 512, -0.5))
    d.record()
    d.synchronize()
    out["c0_2d_single_theta_f64"] = {"points": 262144, "fwd_ms": a.elapsed_time(b) / 5, "inv_ms": b.elapsed_time(c) / 5,
                                     "remap_512sq_ms": c.elapsed_time(d) / 5,
                                     "fwd_points_per_s": 262144 / (a.elapsed_time(b) / 5e3)}

    # 3D nC=320 (4x4x4 tess I): forward + adjoint dL/dtheta, L = 0.5||T(x) - y||^2, 8 theta x 64^3 points (FP64)
    sp3 = CpaSpace([0, 0, 0], [1, 1, 1], (4, 4, 4), tess="I", device=dev)
    pr3 = Prior.create(sp3.geo, 0.15, 0.5)
    th3 = torch.as_tensor(pr3.sample(8, rng), device=dev)
    g = (np.arange(64) + 0.5) / 64
    grid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x3 = torch.as_tensor(np.tile(grid, (8, 1)), device=dev)
    with torch.no_grad():
        y3 = transform(torch.as_tensor(pr3.sample(8, rng), device=dev), x3, sp3, **p)

    def fwd_adjoint_ms(scheme):
        t = th3.clone().requires_grad_(True)
        for _ in range(2):
            t.grad = None
            (0.5 * ((transform(t, x3, sp3, scheme=scheme, **p) - y3) ** 2).sum()).backward()
        a, b = ev(), ev()
        a.record()
        t.grad = None
        (0.5 * ((transform(t, x3, sp3, scheme=scheme, **p) - y3) ** 2).sum()).backward()
        b.record()
        b.synchronize()
        return a.elapsed_time(b)

    n3 = x3.shape[0]
    ms_ref, ms_simple = fwd_adjoint_ms("ref"), fwd_adjoint_ms("simple")
    out["c2_3d_fwd_adjoint_f64"] = {"theta": 8, "points_per_theta": 64 ** 3, "d": sp3.d,
                                    "ms_fwd_plus_adjoint": ms_ref,
                                    "points_per_s": n3 / (ms_ref * 1e-3),
                                    "scheme": "calc_T (closed-form steps + sub-step fallback) forward, adjoint along "
                                              "the forward's branches, expm Frechet adjoint per cell",
                                    "midpoint_scheme_ms_fwd_plus_adjoint": ms_simple}
    del x3, y3

    # the configuration's size in FP32: 64 theta x 128^3 grid points (134 M), forward + adjoint, checkpoints
    # within 48 GB (every 4th time step; the others are recomputed)
    sp32 = CpaSpace([0, 0, 0], [1, 1, 1], (4, 4, 4), tess="I", device=dev, precision=torch.float32)
    th32 = torch.as_tensor(pr3.sample(64, rng), device=dev)
    g = ((np.arange(128) + 0.5) / 128).astype(np.float32)
    grid = torch.as_tensor(np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3), device=dev)
    x32 = grid.repeat(64, 1)
    with torch.no_grad():
        y32 = transform(torch.as_tensor(pr3.sample(64, rng), device=dev), x32, sp32, **p)
    budget = 48 << 30

    def step32():
        t = th32.clone().requires_grad_(True)
        (0.5 * ((transform(t, x32, sp32, memory_budget_bytes=budget, **p) - y32).double() ** 2).sum()).backward()
        return t.grad

    step32()
    a, b = ev(), ev()
    a.record()
    step32()
    b.record()
    b.synchronize()
    ms32 = a.elapsed_time(b)
    out["c2_3d_fwd_adjoint_f32_64theta_128cube"] = {
        "theta": 64, "points_per_theta": 128 ** 3, "d": sp3.d, "ms_fwd_plus_adjoint": ms32,
        "points_per_s": x32.shape[0] / (ms32 * 1e-3),
        "scheme": "calc_T in FP32 (compensated state) forward, its adjoint; gradient FP64",
        "checkpoint_budget_bytes": budget}
    del x32, y32, grid

    # batched MCMC registration: 256 chains x 256^2, FP32, steps captured in a CUDA graph
    sp2 = CpaSpace([0, 0], [1, 1], (4, 4), tess="I", device=dev, precision=torch.float32)
    pr2 = Prior.create(sp2.geo, 0.1, 1.0)
    C, H = 256, 256
    src = np.stack([gaussian_filter(rng.uniform(0, 1, (H, H)).astype(np.float32), 8.0) for _ in range(C)])
    srcg = torch.as_tensor(src, device=dev)
    warped = torch.empty_like(srcg)
    GaussianLogLikelihood(sp2, srcg, srcg, 0.05, p).batch(torch.as_tensor(pr2.sample(C, rng), device=dev),
                                                          warped=warped)
    dst = warped + 0.02 * torch.randn_like(warped)
    ll = GaussianLogLikelihood(sp2, srcg, dst, 0.05, p)
    mh = BatchedMetropolis(ll, torch.zeros((C, sp2.d), device=dev), np.sqrt(np.diag(pr2.cov_cpa)), scale=0.05, seed=3)
    mh.run(10, graph_steps=10)
    torch.cuda.synchronize()
    a, b = ev(), ev()
    a.record()
    mh.run(20, graph_steps=10)
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b) / 20
    out["c3_mcmc_256chains_256sq_f32"] = {"ms_per_mh_step": ms, "mh_steps_per_s_all_chains": C / (ms * 1e-3),
                                          "pixels_per_s": C * H * H / (ms * 1e-3),
                                          "accept_pct_mean": float(mh.accept_ratio().mean())}

    out["remap_ssd_256x256sq_f32_map"] = remap_ssd_c3(torch, dev, mh.theta, srcg, dst)
    return out


# Algorithmic FP32 operation counts of the reference scheme (2D tess I):
# cell lookup 24, affine map M = 2 D^2 = 8; a kept step costs two lookups and
# one map, a midpoint sub-step one lookup, two maps and 4 D axpy operations.
C_CELL_2D, M_2D = 24, 8


def flops_ref_2d(cnt) -> float:
    steps = float(cnt[0] + cnt[1])
    return steps * (2 * C_CELL_2D + M_2D) + float(cnt[2]) * (C_CELL_2D + 2 * M_2D + 4 * 2)


def bench_2d(args, torch, dev, exact: bool = False) -> dict:
    """FP32, batched, on 2D tess I 4x4 (nC=64): 4096 theta x 8192 uniform
    points (268 MB in, larger than L2), through the reference scheme or
    (exact=True) the exact scheme (hitting times), with the error against the
    FP64 oracle of the same scheme on 4 instances."""
    from cpabdiffeo_b200 import _lib, autotune
    from cpabdiffeo_b200.cpa_space import CpaSpace
    from cpabdiffeo_b200.space import Prior
    sp = CpaSpace([0, 0], [1, 1], (4, 4), tess="I", device=dev, precision=torch.float32)
    rng = np.random.default_rng(0)
    nth, npt = 4096, 8192
    theta = torch.as_tensor(Prior.create(sp.geo, 0.1, 1.0).sample(nth, rng), device=dev)
    x = torch.as_tensor(rng.uniform(0, 1, size=(nth * npt, 2)), dtype=torch.float32, device=dev)
    out = torch.empty_like(x)
    p = dict(dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    scheme = _lib.SCHEME_EXACT if exact else _lib.SCHEME_REF
    tuned = autotune.tune(sp, sp.tables_from_theta(theta, DT, 1), x, None, scheme, sample_points=1 << 22, **p)
    stream = torch.cuda.current_stream()
    k_ev = []

    def step(record=False):
        tables = sp.tables_from_theta(theta, DT, 1)
        if record:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
        sp.calc_T_batched(tables, x, out, scheme=scheme, **p)
        if record:
            b.record(stream)
            k_ev.append((a, b))

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index or 0) as clk:
        torch.cuda.nvtx.range_push("timed")
        s.record(stream)
        for _ in range(args.steps):
            step(record=True)
        e.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = s.elapsed_time(e)
    kern_ms = float(np.mean([a.elapsed_time(b) for a, b in k_ev]))
    n = nth * npt
    cnt = torch.zeros(_lib.CNT_N, dtype=torch.int64, device=dev)
    sp.calc_T_batched(sp.tables_from_theta(theta, DT, 1), x, out, counters=cnt, scheme=scheme, **p)
    cnt_h = cnt.cpu().numpy()
    flops = flops_ref_2d(cnt_h)
    peaks = measured_peaks(torch)
    achieved = flops / (kern_ms * 1e-3) / 1e12
    # error against the FP64 oracle of the reference scheme on the first 4 instances
    from oracle import oracle as O
    t = O.tess_struct(2, sp.geo.tess_code, sp.geo.nCs, sp.geo.incs)
    F, nb = O.cell_facets(t, sp.geo.cells)
    out_h, x_h, th_h = out.cpu().numpy(), x.cpu().numpy(), theta.cpu().numpy()
    err = err_fine = 0.0
    for i in range(4):
        A = (sp.geo.B @ th_h[i]).reshape(sp.nC, 6)
        sAo, Tro = O.expm_cells(2, A, DT, 1)
        sl = slice(i * npt, (i + 1) * npt)
        xi = x_h[sl].astype(np.float64)
        if exact:
            ref, _ = O.calc_T_exact(t, Tro, sAo, F, nb, xi, DT, NT, NODE)
        else:
            ref, _ = O.calc_T(t, Tro, sAo, xi, DT, NT, NODE)
        fine, _ = O.calc_T(t, Tro, sAo, xi, DT, NT, 10000)
        err = max(err, float(np.abs(out_h[sl].astype(np.float64) - ref).max()))
        err_fine = max(err_fine, float(np.abs(out_h[sl].astype(np.float64) - fine).max()))
    return {"metric": METRIC, "value": n * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded prior draws, uniform points)",
            "config": {"workload": "batched_2d_tessI_4x4_nc64_4096theta_x_8192pts",
                       "scheme": "exact (facet hitting times)" if exact else "reference calc_T",
                       "dt": DT, "nTimeSteps": NT, "nStepsODE": NODE,
                       "l2": "inputs larger than L2 (268 MB of points)"},
            "gpu_launches": 2 * args.steps, "clocks": clk.summary(), "launch": tuned,
            "work": {"kept_steps": int(cnt_h[0]), "fallback_steps": int(cnt_h[1]), "substeps": int(cnt_h[2]),
                     "points": int(cnt_h[3]), "crossings": int(cnt_h[_lib.CNT_CROSSINGS])},
            "roofline": {"bound": "fp32", "kernel": f"k_integrate<2, tess I, float, {'exact' if exact else 'ref'}>",
                         "achieved": achieved,
                         "peak": peaks["fp32_simt_tflops"], "unit": "TFLOP/s",
                         "frac": achieved / peaks["fp32_simt_tflops"],
                         "peak_source": "measured here: cuBLAS SGEMM 8192^3, TF32 off",
                         "flop_model": f"per step 2*{C_CELL_2D}+{M_2D}, per midpoint sub-step "
                                       f"{C_CELL_2D}+2*{M_2D}+8 (algorithmic, before compensation)",
                         "kernel_ms": kern_ms, "algorithmic_flop_per_launch": flops,
                         "traffic": TRAFFIC_2D_BYTES_PER_LAUNCH},
            "error_vs_fp64_oracle": {"max_abs": err, "points_checked": 4 * npt, "tolerance": 1e-5,
                                     "oracle": "exact scheme (oracle/cpab_oracle_exact.c)" if exact
                                     else "reference scheme (calc_T restated)",
                                     "max_abs_vs_ref_scheme_nODE_1e4": err_fine}}


def remap_ssd_c3(torch, dev, theta, src, dst, reps: int = 10) -> dict:
    """Standalone remap + SSD at the MCMC scale: C FP32 maps [256^2, 2]
    (the inverse transforms of theta [C, d] applied to the pixel centres),
    src and dst [C, 256, 256] float32; 16 algorithmic bytes per pixel (map 8,
    src 4, dst 4); a 256 MB buffer is written before each timed call."""
    from cpabdiffeo_b200.cpa_space import CpaSpace
    from cpabdiffeo_b200.registration import remap_ssd
    from cpabdiffeo_b200.space import pixel_centers
    C, H, W = src.shape
    p = dict(dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    sp2d = CpaSpace([0, 0], [1, 1], (4, 4), tess="I", device=dev, precision=torch.float32)
    xs = torch.as_tensor(pixel_centers(H, W), dtype=torch.float32, device=dev)
    tab = sp2d.tables_from_theta(theta, DT, -1)
    maps = torch.empty((C * H * W, 2), dtype=torch.float32, device=dev)
    offs = torch.arange(C + 1, dtype=torch.int64, device=dev) * (H * W)
    sp2d.calc_T_batched(tab, xs.repeat(C, 1), maps, offsets=offs, **p)
    maps = maps.view(C, H * W, 2)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    pm = (W, -0.5, H, -0.5)
    for _ in range(3):
        remap_ssd(maps, src, dst, 0.05, pixel_map=pm)
    times = []
    torch.cuda.nvtx.range_push("timed_remap")
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        remap_ssd(maps, src, dst, 0.05, pixel_map=pm)
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    torch.cuda.nvtx.range_pop()
    ms_r = float(np.median(times))
    nbytes = 16 * C * H * W
    pk = measured_peaks(torch).get("hbm_gbs")
    ach = nbytes / (ms_r * 1e-3) / 1e9
    return {"ms": ms_r, "images": C, "side": H, "algorithmic_bytes": nbytes, "achieved_gbs": ach,
            "hbm_peak_gbs": pk, "frac": ach / pk if pk else None,
            "l2": "256 MB buffer written before each timed call"}


def bench_mcmc_c3(args, torch, dev) -> dict:
    """Batched MCMC registration (the 256-chain configuration): 256 chains, each
    its own 256x256 FP32 image pair (target = source warped by a prior draw plus
    N(0, 0.02^2) noise), sigma 0.05, random-walk proposals 0.05 Sigma^1/2; a step
    is one Metropolis step of every chain (propose, A = B theta and expm,
    fused integration + remap + SSD, accept), 10 steps per CUDA graph."""
    from scipy.ndimage import gaussian_filter

    from cpabdiffeo_b200 import _lib
    from cpabdiffeo_b200.cpa_space import CpaSpace
    from cpabdiffeo_b200.mcmc import BatchedMetropolis
    from cpabdiffeo_b200.registration import GaussianLogLikelihood
    from cpabdiffeo_b200.space import Prior
    rng = np.random.default_rng(2)
    torch.manual_seed(2)
    p = dict(dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    sp = CpaSpace([0, 0], [1, 1], (4, 4), tess="I", device=dev, precision=torch.float32)
    pr = Prior.create(sp.geo, 0.1, 1.0)
    C, H = 256, 256
    src = torch.as_tensor(np.stack([gaussian_filter(rng.uniform(0, 1, (H, H)).astype(np.float32), 8.0)
                                    for _ in range(C)]), device=dev)
    warped = torch.empty_like(src)
    GaussianLogLikelihood(sp, src, src, 0.05, p).batch(torch.as_tensor(pr.sample(C, rng), device=dev), warped=warped)
    dst = warped + 0.02 * torch.randn_like(warped)
    ll = GaussianLogLikelihood(sp, src, dst, 0.05, p)
    mh = BatchedMetropolis(ll, torch.zeros((C, sp.d), device=dev), np.sqrt(np.diag(pr.cov_cpa)), scale=0.05, seed=3)
    steps = 10 * max(1, -(-args.steps // 10))
    mh.run(10 * max(1, -(-args.warmup // 10)), graph_steps=10)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index or 0) as clk:
        torch.cuda.nvtx.range_push("timed_mcmc")
        s.record()
        mh.run(steps, graph_steps=10)
        e.record()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = s.elapsed_time(e) / steps
    # the fused likelihood kernel alone on the chains' current proposals, with its work counters
    cnt = torch.zeros(_lib.CNT_N, dtype=torch.int64, device=dev)
    ll.batch_tables((mh.sA, mh.Tr), ll=mh.ll_prop, counters=cnt)
    ks, ke = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ks.record()
    for _ in range(5):
        ll.batch_tables((mh.sA, mh.Tr), ll=mh.ll_prop)
    ke.record()
    torch.cuda.synchronize()
    kern_ms = ks.elapsed_time(ke) / 5
    cnt_h = cnt.cpu().numpy()
    flops = flops_ref_2d(cnt_h)
    peaks = measured_peaks(torch)
    achieved = flops / (kern_ms * 1e-3) / 1e12
    return {"metric": METRIC, "value": C * H * H / (ms * 1e-3), "unit": "pixels/s", "n_gpus": 1,
            "steps": steps, "warmup": 10 * max(1, -(-args.warmup // 10)), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (smoothed noise images, targets warped by prior draws plus noise)",
            "config": {"workload": "mcmc_registration_256chains_256x256_f32", "sigma": 0.05, "proposal_scale": 0.05,
                       "graph_steps": 10, "l2": "images 128 MB (src+dst), each step reads all of them"},
            "mh_steps_per_s_all_chains": C / (ms * 1e-3), "accept_pct_mean": float(mh.accept_ratio().mean()),
            "gpu_launches": 4 * steps, "clocks": clk.summary(),
            "work": {"kept_steps": int(cnt_h[0]), "fallback_steps": int(cnt_h[1]), "substeps": int(cnt_h[2]),
                     "pixels": int(cnt_h[3])},
            "roofline": {"bound": "fp32", "kernel": "k_register_ll<tess I, float>", "achieved": achieved,
                         "peak": peaks["fp32_simt_tflops"], "unit": "TFLOP/s",
                         "frac": achieved / peaks["fp32_simt_tflops"],
                         "peak_source": "measured here: cuBLAS SGEMM 8192^3, TF32 off",
                         "flop_model": "the integration's algorithmic FLOPs as for the 2D workload (sampling and SSD "
                                       "not counted)",
                         "kernel_ms": kern_ms, "algorithmic_flop_per_launch": flops, "traffic": None}}


def bench_remap(args, torch, dev) -> dict:
    """remap + SSD of 256 image pairs 256x256 through precomputed FP32 maps."""
    from scipy.ndimage import gaussian_filter

    from cpabdiffeo_b200.space import Prior, build_space
    rng = np.random.default_rng(3)
    C, H = 256, 256
    geo = build_space(2, (4, 4), "I")
    theta = torch.as_tensor(Prior.create(geo, 0.1, 1.0).sample(C, rng), device=dev)
    src = torch.as_tensor(np.stack([gaussian_filter(rng.uniform(0, 1, (H, H)).astype(np.float32), 8.0)
                                    for _ in range(C)]), device=dev)
    dst = src + 0.02 * torch.randn_like(src)
    with ClockSampler(dev.index or 0) as clk:
        r = remap_ssd_c3(torch, dev, theta, src, dst, reps=max(args.steps, 3))
    px = C * H * H
    return {"metric": METRIC, "value": px / (r["ms"] * 1e-3), "unit": "pixels/s", "n_gpus": 1,
            "steps": max(args.steps, 3), "warmup": 3, "ms_per_step": r["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (smoothed noise images)",
            "config": {"workload": "remap_ssd_256images_256x256_f32_maps", "l2": r["l2"]},
            "gpu_launches": 2 * max(args.steps, 3), "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "kernel": "k_remap_ssd_bulk<float> + k_sum_partials", "achieved": r["achieved_gbs"],
                         "peak": r["hbm_peak_gbs"], "unit": "GB/s", "frac": r["frac"],
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                         "bytes_per_pixel": 16, "traffic": TRAFFIC_REMAP_BYTES_PER_LAUNCH}}


def spawn_ranks(n: int) -> int:
    """`bench.py --gpus N` started without a launcher: run this script under
    torch.distributed.run with N local ranks (rendezvous on 127.0.0.1) and
    return its exit status; rank 0 prints the line."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.call(cmd)


def serving_legs(args, dev) -> dict:
    """The serving mix: the capacity one GPU has for it (service times per
    request type: the device-time bound, and the rate the server's job caps
    sustain), the mix at 200 req/s, at 80 % of the lower capacity for
    --serve-sustained-seconds, and at the configuration's 2000 req/s for
    --serve-seconds (above capacity: the server keeps serving transforms while
    registrations queue)."""
    from cpabdiffeo_b200.serving_load import capacity_estimate, make_requests, run_load
    mix = ("1D/2D/3D, nC in {16,64,256,1024}, 1e3-4e6 pts, 10% 200-step registrations (side 64-1024)")
    out = {"serving_capacity": capacity_estimate(device=dev)}
    reqs = make_requests(200.0, 4.0, seed=5)
    out["serving_200hz"] = dict(run_load(reqs, device=dev), arrival_rate_hz=200.0, arrivals_s=4.0)
    cap = min(out["serving_capacity"]["capacity_req_per_s"], out["serving_capacity"]["capacity_with_job_caps"])
    if args.serve_sustained_seconds > 0:
        rate = 0.8 * cap
        reqs = make_requests(rate, args.serve_sustained_seconds, seed=6)
        out["serving_sustained"] = dict(run_load(reqs, device=dev, time_limit_s=4 * args.serve_sustained_seconds + 60),
                                        arrival_rate_hz=rate, arrivals_s=args.serve_sustained_seconds, mix=mix)
    reqs = make_requests(2000.0, args.serve_seconds, seed=4)
    out["serving"] = dict(run_load(reqs, device=dev, grace_s=1.0), arrival_rate_hz=2000.0,
                          arrivals_s=args.serve_seconds, mix=mix,
                          window="arrivals + 1 s; what is still queued or running then is reported, not waited for")
    return out


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist

    from cpabdiffeo_b200 import _lib
    from cpabdiffeo_b200.cpa_space import CpaSpace

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.workload != "batched_1d":
        line = {"batched_2d_nc64": bench_2d, "remap_ssd": bench_remap, "mcmc_c3": bench_mcmc_c3,
                "exact_2d_nc64": lambda a, t, d: bench_2d(a, t, d, exact=True),
                "serving": lambda a, t, d: serving_legs(a, d)}[args.workload](args, torch, dev)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    geo, theta_h, sizes, offsets_h, pts_h = make_workload(rank, args.theta)
    n_total = int(offsets_h[-1])
    sp = CpaSpace([0.0], [1.0], (NC,), device=dev, precision=torch.float32)
    theta = torch.as_tensor(theta_h, device=dev)
    offsets = torch.as_tensor(offsets_h, device=dev)
    pts = torch.as_tensor(pts_h, device=dev)
    out = torch.empty_like(pts)
    p = dict(dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    from cpabdiffeo_b200 import autotune
    tuned = autotune.tune(sp, sp.tables_from_theta(theta, DT, 1), pts, offsets, _lib.SCHEME_EXACT, **p)
    # the step (prologue + tile prefix + integration) captured once in a CUDA graph, replayed per step
    graph_step = sp.capture_batched(args.theta, pts, out, offsets=offsets, scheme=_lib.SCHEME_EXACT, **p)
    graph_step.theta.copy_(theta)
    k_ev = []

    def step(record=False):
        if record:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
        graph_step()
        if record:
            b.record(stream)
            k_ev.append((a, b))

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed")      # lets a profiler select the timed launches by name
        s.record(stream)
        for _ in range(args.steps):
            step(record=True)
        e.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    barrier()
    ms = s.elapsed_time(e)
    step_ms = float(np.mean([a.elapsed_time(b) for a, b in k_ev]))
    from cpabdiffeo_b200.distributed import max_over_ranks
    ms = max_over_ranks(ms, dev)
    value = n_total * world * args.steps / (ms * 1e-3)
    out_dev_h = out.cpu().numpy()

    # the integration kernel alone (the graph's other two launches are a few microseconds): eager launches
    # on the same buffers, timed with events on the launching stream
    tables = sp.tables_from_theta(theta, DT, 1)
    ws = torch.empty(int(sp._ctx.lib.cpab_batched_workspace_bytes(args.theta)), dtype=torch.uint8, device=dev)

    def kernel_ms(offs, n_uniform=0, reps=5):
        kt = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            if offs is None:
                sp.calc_T_batched(tables, pts[:n_uniform * args.theta], out[:n_uniform * args.theta],
                                  scheme=_lib.SCHEME_EXACT, **p)
            else:
                sp.calc_T_batched(tables, pts, out, offsets=offs, workspace=ws, scheme=_lib.SCHEME_EXACT, **p)
            b.record(stream)
            kt.append((a, b))
        torch.cuda.synchronize()
        return float(np.median([a.elapsed_time(b) for a, b in kt]))

    kern_ms = kernel_ms(offsets)
    # load balance of the ragged batch: the same instances with equal point counts (same total up to
    # rounding) in a uniform launch
    n_eq = n_total // args.theta
    uniform_ms = kernel_ms(None, n_uniform=n_eq)
    load_balance = {"ragged_points_per_s": n_total / (kern_ms * 1e-3),
                    "uniform_points_per_s": n_eq * args.theta / (uniform_ms * 1e-3),
                    "achieved_over_ideal": (n_total / kern_ms) / (n_eq * args.theta / uniform_ms)}

    # end to end through the public API, host buffers (pinned), copies inside the timed region
    pts_pin = torch.from_numpy(pts_h).pin_memory()
    out_pin = torch.empty_like(pts_pin).pin_memory()
    th_pin = torch.from_numpy(theta_h).pin_memory()

    def e2e_step():
        # the public host-buffer entry point: chunked copy-in / integrate / copy-out on three streams
        sp.calc_T_batched_host(th_pin, pts_pin, out_pin, offsets_h, mysign=1, scheme=_lib.SCHEME_EXACT,
                               chunks=args.e2e_chunks, **p)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e2.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = s2.elapsed_time(e2)
    ms_e2e = max_over_ranks(ms_e2e, dev)
    h2d = pts_h.nbytes + theta_h.nbytes + offsets_h.nbytes
    d2h = pts_h.nbytes
    # the host-buffer result must equal the device-resident one (same inputs, same kernels)
    e2e_equal = bool(np.array_equal(out_pin.numpy(), out_dev_h))

    # the host link alone: the same bytes copied in and out concurrently on two streams (no compute);
    # the end-to-end figure cannot beat n_total / this time
    s_a, s_b = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    link_ms = []
    for _ in range(3):
        torch.cuda.synchronize()
        la, lb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        la.record(stream)
        s_a.wait_stream(stream)
        s_b.wait_stream(stream)
        with torch.cuda.stream(s_a):
            pts.copy_(pts_pin, non_blocking=True)
        with torch.cuda.stream(s_b):
            out_pin.copy_(out, non_blocking=True)
        stream.wait_stream(s_a)
        stream.wait_stream(s_b)
        lb.record(stream)
        lb.synchronize()
        link_ms.append(la.elapsed_time(lb))
    link_ms = min(link_ms)

    # work accounting (counters) of the timed scheme
    cnt = torch.zeros(_lib.CNT_N, dtype=torch.int64, device=dev)
    sp.calc_T_batched(tables, pts, out, offsets=offsets, workspace=ws, counters=cnt, scheme=_lib.SCHEME_EXACT, **p)
    torch.cuda.synchronize()
    cnt_h = cnt.cpu().numpy()
    flops = flops_exact(cnt_h)

    # the same workload with FP64 points (the configuration names both precisions)
    sp64 = CpaSpace([0.0], [1.0], (NC,), device=dev, precision=torch.float64)
    pts64 = pts.double()
    out64 = torch.empty_like(pts64)
    autotune.tune(sp64, sp64.tables_from_theta(theta, DT, 1), pts64, offsets, _lib.SCHEME_EXACT, **p)
    g64 = sp64.capture_batched(args.theta, pts64, out64, offsets=offsets, scheme=_lib.SCHEME_EXACT, **p)
    g64.theta.copy_(theta)
    for _ in range(3):
        g64()
    torch.cuda.synchronize()
    s4, e4 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s4.record(stream)
    for _ in range(args.steps):
        g64()
    e4.record(stream)
    torch.cuda.synchronize()
    ms64 = max_over_ranks(s4.elapsed_time(e4), dev) / args.steps
    out64_h = out64.cpu().numpy()
    del pts64, out64, g64

    # the same workload through the reference's REF scheme (FP32 on the GPU), its own tuned launch shape
    sp_ref = CpaSpace([0.0], [1.0], (NC,), device=dev, precision=torch.float32)
    tab_ref = sp_ref.tables_from_theta(theta, DT, 1)
    tuned_ref = autotune.tune(sp_ref, tab_ref, pts, offsets, _lib.SCHEME_REF, sample_points=2_000_000, **p)
    cnt_ref = torch.zeros(_lib.CNT_N, dtype=torch.int64, device=dev)
    sp_ref.calc_T_batched(tab_ref, pts, out, offsets=offsets, workspace=ws, scheme=_lib.SCHEME_REF,
                          counters=cnt_ref, **p)
    torch.cuda.synchronize()
    s3, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_ref_steps = 2
    torch.cuda.nvtx.range_push("timed_ref")
    s3.record(stream)
    for _ in range(n_ref_steps):
        sp_ref.calc_T_batched(tab_ref, pts, out, offsets=offsets, workspace=ws, scheme=_lib.SCHEME_REF, **p)
    e3.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    ms_ref = s3.elapsed_time(e3) / n_ref_steps
    out_ref_h = out.cpu().numpy()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded prior draws, log-uniform ragged sizes, uniform points)",
            "config": {"workload": WORKLOAD, "n_theta_per_gpu": args.theta, "points_per_gpu": n_total,
                       "nC": NC, "integration_time": 1.0,
                       "scheme": "closed form across cells (ClosedFormInt restated: hitting times in FP64)",
                       "precision": "f32 points, f64 hitting times and expm",
                       "step": "CUDA graph replay: theta -> A -> expm prologue, tile prefix, persistent integration",
                       "l2": "inputs larger than L2 (352 MB of points per GPU)",
                       "parallelism": f"independent shards x{world}"},
            "e2e": {"value": n_total * world * args.steps / (ms_e2e * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "result_equals_device_run": e2e_equal,
                    "link_only_ms": link_ms,
                    "link_bound_points_per_s": n_total * world / (link_ms * 1e-3),
                    "pipeline": f"{args.e2e_chunks} instance groups (1/4, 1/2, 1, ..., 1, 1/2, 1/4 of the points), "
                                "3 streams (copy in / integrate / copy out), pinned host buffers"},
            "gpu_launches": 3 * args.steps,
            "clocks": clk.summary(),
            "work": {"cell_visits": int(cnt_h[0]), "points": int(cnt_h[3]), "failed": int(cnt_h[4])},
            "load_balance": load_balance,
            "fp64": {"value": n_total * world / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64,
                     "precision": "f64 points and arithmetic"},
            "ref_scheme_gpu": {"points_per_s": n_total * world / (ms_ref * 1e-3), "ms_per_step": ms_ref,
                               "precision": "f32", "scheme": "reference calc_T dt=0.02 nT=50 nODE=100",
                               "launch": tuned_ref},
            "launch": tuned}
    if rank == 0:
        peaks = measured_peaks(torch)
        achieved = flops / (kern_ms * 1e-3) / 1e12
        line["roofline"] = {"bound": "fp64", "kernel": "k_exact1d<float>", "achieved": achieved,
                            "peak": peaks["fp64_tflops"], "unit": "TFLOP/s",
                            "frac": achieved / peaks["fp64_tflops"],
                            "peak_source": "measured here: cuBLAS DGEMM 4096^3",
                            "flop_model": f"{EXACT_FLOP_PER_VISIT} per cell visit + {EXACT_FLOP_PER_POINT} per point "
                                          "(log/exp counted as 20)",
                            "kernel_ms": kern_ms, "step_ms_events": step_ms,
                            "traffic": TRAFFIC_EXACT1D_BYTES_PER_POINT * n_total,
                            "traffic_note": "ncu DRAM bytes of one launch on the 2048-theta case, scaled by points",
                            "pipes_ncu": PIPES_EXACT1D,
                            "algorithmic_flop_per_launch": flops,
                            "hbm_achieved_gbs": 2 * pts_h.nbytes / (kern_ms * 1e-3) / 1e9,
                            "hbm_peak_gbs": peaks.get("hbm_gbs")}
        flops_ref = flops_from_counters(cnt_ref.cpu().numpy(), 1)
        ach_ref = flops_ref / (ms_ref * 1e-3) / 1e12
        line["ref_scheme_gpu"]["roofline"] = {
            "bound": "fp32", "kernel": "k_integrate<1, float, ref>", "achieved": ach_ref,
            "peak": peaks["fp32_simt_tflops"], "unit": "TFLOP/s", "frac": ach_ref / peaks["fp32_simt_tflops"],
            "peak_source": "measured here: cuBLAS SGEMM 8192^3, TF32 off",
            "flop_model": "per step 2*5+2, per midpoint sub-step 5+2*2+4 (algorithmic)"}
        # errors: the timed FP32 result and the FP64 run against the FP64 closed form (oracle) on 64
        # instances; both GPU schemes against the reference's calc_T scheme in FP64 on 8
        from oracle import oracle as O
        rel32 = rel64 = abs32 = 0.0
        n_cf = 0
        for i in range(min(64, args.theta)):
            A = (geo.B @ theta_h[i]).reshape(NC, 2)
            sl = slice(offsets_h[i], offsets_h[i + 1])
            x = pts_h[sl].astype(np.float64)[:, 0]
            ref, _ = O.closed_form_1d(A, NC, x, DT * NT)
            g32 = out_dev_h[sl].astype(np.float64)[:, 0]
            den = np.maximum(np.abs(ref), 1e-6)
            rel32 = max(rel32, float((np.abs(g32 - ref) / den).max()))
            abs32 = max(abs32, float(np.abs(g32 - ref).max()))
            rel64 = max(rel64, float((np.abs(out64_h[sl][:, 0] - ref) / den).max()))
            n_cf += x.size
        line["error_vs_fp64_closed_form"] = {
            "max_rel_f32": rel32, "max_abs_f32": abs32, "max_rel_f64": rel64, "instances_checked": min(64, args.theta),
            "points_checked": n_cf, "tolerance_rel_f32": 1e-5, "tolerance_f64": 1e-12,
            "relative_to": "max(|closed form|, 1e-6)"}
        line["fp64"]["max_rel_error_vs_closed_form"] = rel64
        t = O.tess_struct(1, 2, geo.nCs, geo.incs)
        err_exact = err_ref = 0.0
        n_chk = 0
        for i in range(8):
            A = (geo.B @ theta_h[i]).reshape(NC, 2)
            sAo, Tro = O.expm_cells(1, A, DT, 1)
            sl = slice(offsets_h[i], offsets_h[i + 1])
            x = pts_h[sl].astype(np.float64)
            ref, _ = O.calc_T(t, Tro, sAo, x, DT, NT, NODE)
            ref = O.clamp_1d(ref)
            err_exact = max(err_exact, float(np.abs(out_dev_h[sl].astype(np.float64) - ref).max()))
            err_ref = max(err_ref, float(np.abs(out_ref_h[sl].astype(np.float64) - ref).max()))
            n_chk += x.shape[0]
        line["error_vs_fp64_reference_scheme"] = {"max_abs_closed_form_f32": err_exact,
                                                  "max_abs_ref_scheme_f32": err_ref,
                                                  "points_checked": n_chk,
                                                  "note": "the closed form is the exact flow the reference's "
                                                          "step scheme approximates"}
        if world == 1 and not args.no_extras:
            r, sample, kind, cores, _ = cpu_reference_rate(theta_h, offsets_h, pts_h, geo, 400_000)
            line["cpu_baseline"] = {"value": r, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
                                    "scheme": "the reference's calc_T (its own CPU-compiled kernel source, FP64)"}
            r2, sample2, cores2 = cpu_closed_form_rate(theta_h, offsets_h, pts_h, geo, 4_000_000)
            line["cpu_baseline_same_scheme"] = {
                "value": r2, "unit": UNIT, "cores": cores2, "kind": "port", "sample": sample2,
                "scheme": "closed form (ClosedFormInt restated in C, pinned to the reference's calc_phi), FP64",
                "gpu_over_cpu_device": value / r2, "gpu_over_cpu_e2e": line["e2e"]["value"] / r2}
            try:
                line["plain_vs_batched_2d"] = plain_vs_batched_2d(torch, dev)
            except Exception as ex:  # reported, never fatal
                line["plain_vs_batched_2d"] = {"error": repr(ex)}
            for key, ex_flag in (("batched_2d_ref_f32", False), ("batched_2d_exact_f32", True)):
                try:
                    line[key] = bench_2d(argparse.Namespace(steps=3, warmup=3), torch, dev, exact=ex_flag)
                    for k in ("metric", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data"):
                        line[key].pop(k, None)
                except Exception as ex:
                    line[key] = {"error": repr(ex)}
            try:
                line["other_configs"] = other_configs(torch, dev)
            except Exception as ex:
                line["other_configs"] = {"error": repr(ex)}
            if args.serve_seconds > 0:
                try:
                    line.update(serving_legs(args, dev))
                except Exception as ex:
                    line["serving"] = {"error": repr(ex)}
        print(json.dumps(line), flush=True)
    del graph_step
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
