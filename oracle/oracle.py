"""Python access to the CPU parity oracle.  TEST INFRASTRUCTURE ONLY.

Two libraries, both built by oracle/Makefile:
  * liboracle.so      -- this repository's C restatement (cpab_oracle.c),
                         the checker every GPU parity test uses;
  * _ref/libcpab_ref.so -- the reference's own kernel sources compiled as host
                         code (ref_kernels.cpp, ref_expm.cpp); present only where
                         the reference checkout existed at build time.  It pins
                         the restatement (tests/golden/make_golden.py) and serves
                         as the CPU baseline of bench.py when available.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libcpab_ref.so"

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class OracleTess(C.Structure):
    _fields_ = [("dim", C.c_int), ("tess", C.c_int), ("nC0", C.c_int), ("nC1", C.c_int), ("nC2", C.c_int),
                ("inc_x", C.c_double), ("inc_y", C.c_double), ("inc_z", C.c_double)]


def ref_root() -> Path | None:
    """The cpabDiffeo checkout to compile oracle/_ref from: $CPAB_REF_ROOT, else
    the checkout mounted at /root/reference in the build container; None when
    neither exists (the GPU box uses the prebuilt oracle/_ref)."""
    for cand in (os.environ.get("CPAB_REF_ROOT"), "/root/reference"):
        if cand and (Path(cand) / "cpab" / "gpu" / "calc_2Dto2D.cu").exists():
            return Path(cand)
    return None


def build(quiet: bool = True) -> None:
    """Run the oracle Makefile (liboracle.so; _ref only if the reference exists)."""
    root = ref_root()
    args = ["make", "-C", str(HERE)] + ([f"REF_ROOT={root}"] if root else [])
    r = subprocess.run(args, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        print(r.stdout)


_ora = None
_ref = None


def lib() -> C.CDLL:
    global _ora
    if _ora is None:
        if not ORACLE_SO.exists():
            build()
        L = C.CDLL(str(ORACLE_SO))
        L.oracle_cell_idx.restype = C.c_int
        L.oracle_calc_T.restype = C.c_int64
        L.oracle_closed_form_1d.restype = C.c_int64
        L.oracle_remap_ssd.restype = C.c_double
        L.oracle_remap3d_ssd.restype = C.c_double
        _ora = L
    return _ora


def ref_available() -> bool:
    return REF_SO.exists()


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} (built only where the reference sources exist)")
        _ref = C.CDLL(str(REF_SO))
    return _ref


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def tess_struct(dim: int, tess: int, nCs, incs) -> OracleTess:
    n = list(nCs) + [0] * (3 - len(nCs))
    i = list(incs) + [1.0] * (3 - len(incs))
    return OracleTess(dim, tess, n[0], n[1], n[2], i[0], i[1], i[2])


# ------------------------------------------------------------------ restatement


def calc_cell_idx(t: OracleTess, pts) -> np.ndarray:
    pts = _c64(pts)
    out = np.empty(pts.shape[0], dtype=np.int32)
    lib().oracle_calc_cell_idx(C.byref(t), _d(pts), out.ctypes.data_as(_ip), C.c_int64(pts.shape[0]))
    return out


def calc_v(t: OracleTess, As, pts) -> np.ndarray:
    pts, As = _c64(pts), _c64(As)
    out = np.empty_like(pts)
    lib().oracle_calc_v(C.byref(t), _d(As), _d(pts), _d(out), C.c_int64(pts.shape[0]))
    return out


def expm_cells(dim: int, A, dt: float, sign: int):
    """(signedA, Trels) for cells A [..., ne]."""
    A = _c64(A)
    ne = dim * (dim + 1)
    n = A.size // ne
    sA = np.empty_like(A)
    Tr = np.empty_like(A)
    lib().oracle_expm_cells(C.c_int(dim), _d(A), C.c_int64(n), C.c_double(dt), C.c_int(sign), _d(sA), _d(Tr))
    return sA, Tr


def calc_T(t: OracleTess, Trels, sA, pts, dt, nT, nODE):
    """Returns (out, number of fallback steps)."""
    pts = _c64(pts)
    out = np.empty_like(pts)
    nfb = lib().oracle_calc_T(C.byref(t), _d(_c64(Trels)), _d(_c64(sA)), _d(pts), _d(out),
                              C.c_int64(pts.shape[0]), C.c_double(dt), C.c_int(nT), C.c_int(nODE))
    return out, int(nfb)


def calc_T_simple(t: OracleTess, sA, pts, dt, nT, nODE):
    pts = _c64(pts)
    out = np.empty_like(pts)
    lib().oracle_calc_T_simple(C.byref(t), _d(_c64(sA)), _d(pts), _d(out), C.c_int64(pts.shape[0]),
                               C.c_double(dt), C.c_int(nT), C.c_int(nODE))
    return out


def calc_trajectory(t: OracleTess, Trels, sA, pts, dt, nT, nODE):
    pts = _c64(pts)
    traj = np.empty((nT + 1,) + pts.shape)
    lib().oracle_calc_trajectory(C.byref(t), _d(_c64(Trels)), _d(_c64(sA)), _d(pts), _d(traj),
                                 C.c_int64(pts.shape[0]), C.c_double(dt), C.c_int(nT), C.c_int(nODE))
    return traj


def closed_form_1d(sA, nC: int, pts, t_total: float):
    """ClosedFormInt.calc_phi per point on [0,1]; returns (out, n_failed)."""
    sA = _c64(sA).reshape(nC, 2)
    x_tess = np.linspace(0.0, 1.0, nC + 1)
    vel = np.empty(nC + 1)
    for k in range(nC + 1):
        c = min(k, nC - 1)
        vel[k] = sA[c, 0] * x_tess[k] + sA[c, 1]
    pts = _c64(pts).reshape(-1)
    out = np.empty_like(pts)
    nf = lib().oracle_closed_form_1d(_d(sA), _d(x_tess), _d(vel), C.c_int(nC), _d(pts), _d(out),
                                     C.c_int64(pts.size), C.c_double(t_total))
    return out, int(nf)


def cell_facets(t: OracleTess, cells) -> tuple[np.ndarray, np.ndarray]:
    """Facets of every cell (cpab_oracle_exact.c): ([nC, nF, dim+1] rows
    (outward unit normal, -offset), [nC, nF] neighbour cell or -1)."""
    cells = _c64(cells)
    nC, nV, nh = cells.shape
    nF = nh if (nV == nh and t.dim > 1) else 2 * t.dim
    F = np.empty((nC, nF, nh))
    nb = np.empty((nC, nF), dtype=np.int32)
    got = lib().oracle_cell_facets(C.byref(t), _d(cells), C.c_int(nV), _d(F), nb.ctypes.data_as(_ip))
    assert got == nF
    return F, nb


def calc_T_exact(t: OracleTess, Trels, sA, facets, nbr, pts, dt, nT, nODE):
    """EXACT scheme (hitting times; cpab_oracle_exact.c). Returns (out, counters[4]):
    steps kept, steps with an exit, facet crossings, fallbacks."""
    pts = _c64(pts)
    out = np.empty_like(pts)
    cnt = np.zeros(4, dtype=np.int64)
    F = _c64(facets)
    nb = np.ascontiguousarray(nbr, dtype=np.int32)
    lib().oracle_calc_T_exact(C.byref(t), _d(_c64(Trels)), _d(_c64(sA)), _d(F), nb.ctypes.data_as(_ip),
                              C.c_int(F.shape[1]), _d(pts), _d(out), C.c_int64(pts.shape[0]), C.c_double(dt),
                              C.c_int(nT), C.c_int(nODE), cnt.ctypes.data_as(C.POINTER(C.c_int64)))
    return out, cnt


def clamp_1d(x, lo=0.0, hi=1.0):
    """threshold_krnl (cpab/cpaNd/_CpaSpace.py:35-43)."""
    y = np.array(x, dtype=np.float64, copy=True)
    y[y < lo] = lo
    y[y > hi] = hi
    return y


# ------------------------------------------------------------------ reference (host-compiled)


def _ref_fn(name):
    return getattr(ref_lib(), name)


def ref_calc_cell_idx(dim: int, tess: int, nCs, incs, pts, nC: int) -> np.ndarray:
    pts = _c64(pts).copy()
    out = np.empty(pts.shape[0], dtype=np.int32)
    n = list(nCs) + [0] * (3 - len(nCs))
    i = list(incs) + [1.0] * (3 - len(incs))
    _ref_fn(f"ref_d{dim}_t{tess}_calc_cell_idx")(_d(pts), out.ctypes.data_as(_ip), C.c_int(pts.shape[0]),
                                                 C.c_int(n[0]), C.c_int(n[1]), C.c_int(n[2]),
                                                 C.c_double(i[0]), C.c_double(i[1]), C.c_double(i[2]), C.c_int(nC))
    return out


def ref_calc_v(dim, tess, nCs, incs, As, pts, nC):
    pts = _c64(pts).copy()
    As = _c64(As).copy()
    vel = np.zeros_like(pts)
    n = list(nCs) + [0] * (3 - len(nCs))
    i = list(incs) + [1.0] * (3 - len(incs))
    _ref_fn(f"ref_d{dim}_t{tess}_calc_v")(_d(pts), _d(vel), _d(As), C.c_int(pts.shape[0]),
                                          C.c_int(n[0]), C.c_int(n[1]), C.c_int(n[2]),
                                          C.c_double(i[0]), C.c_double(i[1]), C.c_double(i[2]), C.c_int(nC))
    return vel


def ref_calc_T(dim, tess, nCs, incs, Trels, sA, pts, dt, nT, nODE, nC, simple=False):
    pts = _c64(pts).copy()
    out = np.zeros_like(pts)
    n = list(nCs) + [0] * (3 - len(nCs))
    i = list(incs) + [1.0] * (3 - len(incs))
    common = [C.c_double(dt), C.c_int(nT), C.c_int(nODE), C.c_int(pts.shape[0]),
              C.c_int(n[0]), C.c_int(n[1]), C.c_int(n[2]),
              C.c_double(i[0]), C.c_double(i[1]), C.c_double(i[2]), C.c_int(nC)]
    if simple:
        _ref_fn(f"ref_d{dim}_t{tess}_calc_T_simple")(_d(pts), _d(out), _d(_c64(sA).copy()), *common)
    else:
        _ref_fn(f"ref_d{dim}_t{tess}_calc_T")(_d(pts), _d(out), _d(_c64(Trels).copy()), _d(_c64(sA).copy()),
                                              *common)
    return out


def ref_calc_trajectory(dim, tess, nCs, incs, Trels, sA, pts, dt, nT, nODE, nC):
    pts = _c64(pts)
    nP = pts.shape[0]
    pos = np.zeros((nT * nP, dim))
    pos[:nP] = pts
    n = list(nCs) + [0] * (3 - len(nCs))
    i = list(incs) + [1.0] * (3 - len(incs))
    _ref_fn(f"ref_d{dim}_t{tess}_calc_trajectory")(_d(pos), _d(_c64(Trels).copy()), _d(_c64(sA).copy()),
                                                   C.c_double(dt), C.c_int(nT), C.c_int(nODE), C.c_int(nP),
                                                   C.c_int(n[0]), C.c_int(n[1]), C.c_int(n[2]),
                                                   C.c_double(i[0]), C.c_double(i[1]), C.c_double(i[2]),
                                                   C.c_int(nC))
    return np.concatenate([pts[None], pos.reshape(nT, nP, dim)], axis=0)


def ref_expm(dim: int, M) -> np.ndarray:
    """The reference's gpu_expm kernel (p=12) on dt-scaled signed matrices M [n, ne]."""
    M = _c64(M).copy()
    ne = dim * (dim + 1)
    n = M.size // ne
    T = np.zeros_like(M)
    _ref_fn(f"ref_expm{dim}d")(_d(M), _d(T), C.c_int(n), C.c_int(12))
    return T


def ref_expm_1d(M) -> np.ndarray:
    """The reference's 1D closed form (cpab/cpaNd/_CpaCalcs.py:285-292), numpy as there."""
    M = _c64(M).reshape(-1, 2)
    T = np.empty_like(M)
    np.exp(M[:, 0], out=T[:, 0])
    T[:, 1] = M[:, 1]
    idx = M[:, 0] != 0
    T[idx, 1] = T[idx, 1] * (T[idx, 0] - 1) / M[idx, 0]
    return T


def remap(map_pts, src, sx, ox, sy, oy) -> np.ndarray:
    """warped [H, W] float64 from a map [H*W, 2] and a float32 image [H, W]."""
    src = np.ascontiguousarray(src, dtype=np.float32)
    H, W = src.shape
    mp = _c64(map_pts)
    out = np.empty(H * W)
    lib().oracle_remap(_d(mp), src.ctypes.data_as(_fp), _d(out), C.c_int(H), C.c_int(W), C.c_double(sx),
                       C.c_double(ox), C.c_double(sy), C.c_double(oy))
    return out.reshape(H, W)


def remap_ssd(map_pts, src, dst, sigma, sx, ox, sy, oy):
    """(ll, warped) with ll = sum -0.5 (warped - dst)^2 / sigma^2 (Kahan sum)."""
    src = np.ascontiguousarray(src, dtype=np.float32)
    dst = np.ascontiguousarray(dst, dtype=np.float32)
    H, W = src.shape
    mp = _c64(map_pts)
    warped = np.empty(H * W)
    ll = lib().oracle_remap_ssd(_d(mp), src.ctypes.data_as(_fp), dst.ctypes.data_as(_fp), C.c_int(H), C.c_int(W),
                                C.c_double(sx), C.c_double(ox), C.c_double(sy), C.c_double(oy),
                                C.c_double(sigma), _d(warped))
    return float(ll), warped.reshape(H, W)


def remap3d(map_pts, src, sx, ox, sy, oy, sz, oz) -> np.ndarray:
    """warped [H, W, D] float64 from a map [H*W*D, 3] and a float32 volume [H, W, D]
    (cpab_oracle.c oracle_remap3d: img[row][col][slice], trilinear, zero outside)."""
    src = np.ascontiguousarray(src, dtype=np.float32)
    H, W, D = src.shape
    mp = _c64(map_pts)
    out = np.empty(H * W * D)
    lib().oracle_remap3d(_d(mp), src.ctypes.data_as(_fp), _d(out), C.c_int(H), C.c_int(W), C.c_int(D),
                         C.c_double(sx), C.c_double(ox), C.c_double(sy), C.c_double(oy), C.c_double(sz),
                         C.c_double(oz))
    return out.reshape(H, W, D)


def remap3d_ssd(map_pts, src, dst, sigma, sx, ox, sy, oy, sz, oz):
    """(ll, warped) of the trilinear remap, ll = sum -0.5 (warped - dst)^2 / sigma^2 (Kahan sum)."""
    src = np.ascontiguousarray(src, dtype=np.float32)
    dst = np.ascontiguousarray(dst, dtype=np.float32)
    H, W, D = src.shape
    mp = _c64(map_pts)
    warped = np.empty(H * W * D)
    ll = lib().oracle_remap3d_ssd(_d(mp), src.ctypes.data_as(_fp), dst.ctypes.data_as(_fp), C.c_int(H), C.c_int(W),
                                  C.c_int(D), C.c_double(sx), C.c_double(ox), C.c_double(sy), C.c_double(oy),
                                  C.c_double(sz), C.c_double(oz), C.c_double(sigma), _d(warped))
    return float(ll), warped.reshape(H, W, D)


def register_ll(t: OracleTess, Trels_inv, sA_inv, src, dst, sigma, dt, nT, nODE):
    """The registration log-likelihood of one image pair: the pixel centres
    are mapped by T^-1 (tables with sign -1), src is sampled there and scored
    against dst (cpab/cpa2d/model/transformations/register/
    _ScaleDependentLogLikelihoodGaussian.py:34-109)."""
    H, W = np.shape(src)
    ys, xs = np.meshgrid((np.arange(H) + 0.5) / H, (np.arange(W) + 0.5) / W, indexing="ij")
    grid = np.stack([xs.ravel(), ys.ravel()], axis=1)
    pts, _ = calc_T(t, Trels_inv, sA_inv, grid, dt, nT, nODE)
    return remap_ssd(pts, src, dst, sigma, W, -0.5, H, -0.5)


# ------------------------------------------------------------------ MCMC (batched Metropolis)


def philox4x32_10(c, key):
    """Philox4x32-10 (Salmon et al., SC 2011) on uint32 arrays c[..., 4]; key (k0, k1)."""
    M0, M1, W0, W1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57), np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
    mask = np.uint64(0xFFFFFFFF)
    c = [np.asarray(c[..., i], dtype=np.uint64) for i in range(4)]
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    for _ in range(10):
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c = [(hi1 ^ c[1] ^ k0) & mask, lo1, (hi0 ^ c[3] ^ k1) & mask, lo0]
        k0 = (k0 + W0) & mask
        k1 = (k1 + W1) & mask
    return np.stack(c, axis=-1).astype(np.uint32)


def _u53(hi, lo):
    m = (hi.astype(np.uint64) >> np.uint64(5)) << np.uint64(26) | (lo.astype(np.uint64) >> np.uint64(6))
    return (m.astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def mcmc_normals(seed: int, step: int, C: int, d: int) -> np.ndarray:
    """z [C, d] of the proposal at `step` (stream 0), as the GPU draws them."""
    pairs = (d + 1) // 2
    ch, j = np.meshgrid(np.arange(C), np.arange(pairs), indexing="ij")
    c = np.stack([ch, np.full_like(ch, step & 0xFFFFFFFF), np.full_like(ch, ((step >> 32) << 8) | 0), j], -1)
    r = philox4x32_10(c.astype(np.uint64), (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))
    u1, u2 = _u53(r[..., 0], r[..., 1]), _u53(r[..., 2], r[..., 3])
    rad = np.sqrt(-2.0 * np.log(u1))
    z = np.empty((C, 2 * pairs))
    z[:, 0::2] = rad * np.cos(2 * np.pi * u2)
    z[:, 1::2] = rad * np.sin(2 * np.pi * u2)
    return z[:, :d]


def mcmc_local_draws(seed: int, step: int, C: int, nV: int, dim: int):
    """(k [C], z [C, dim]) of the local proposal at `step` (Philox stream 2): the
    vertex from word 0 of counter (chain, step, 2, 0), the normals from
    counters (chain, step, 2, 1 + pair), as the GPU draws them."""
    key = (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    hi = ((step >> 32) << 8) | 2
    ch = np.arange(C)
    c0 = np.stack([ch, np.full_like(ch, step & 0xFFFFFFFF), np.full_like(ch, hi), np.zeros_like(ch)], -1)
    r0 = philox4x32_10(c0.astype(np.uint64), key)
    k = np.minimum((_u53(r0[..., 0], r0[..., 1]) * nV).astype(np.int64), nV - 1)
    z = np.empty((C, 2 * ((dim + 1) // 2)))
    for p in range((dim + 1) // 2):
        c = np.stack([ch, np.full_like(ch, step & 0xFFFFFFFF), np.full_like(ch, hi), np.full_like(ch, 1 + p)], -1)
        r = philox4x32_10(c.astype(np.uint64), key)
        u1, u2 = _u53(r[..., 0], r[..., 1]), _u53(r[..., 2], r[..., 3])
        rad = np.sqrt(-2.0 * np.log(u1))
        z[:, 2 * p] = rad * np.cos(2 * np.pi * u2)
        z[:, 2 * p + 1] = rad * np.sin(2 * np.pi * u2)
    return k, z[:, :dim]


def mcmc_log_uniform(seed: int, step: int, C: int) -> np.ndarray:
    ch = np.arange(C)
    c = np.stack([ch, np.full_like(ch, step & 0xFFFFFFFF), np.full_like(ch, ((step >> 32) << 8) | 1),
                  np.zeros_like(ch)], -1)
    r = philox4x32_10(c.astype(np.uint64), (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))
    return np.log(_u53(r[..., 0], r[..., 1]))


def mcmc_run(B, ll_of_theta, theta0, prop_std, scale, seed, n_steps, inv_npts, rule=0):
    """Batched Metropolis on the CPU with the GPU's random stream.
    ll_of_theta(theta [C, d]) -> [C].  Returns (theta, ll, accepted [n_steps, C])."""
    theta = np.array(theta0, dtype=np.float64, copy=True)
    C, d = theta.shape
    ll = ll_of_theta(theta)
    acc = np.zeros((n_steps, C), dtype=bool)
    for step in range(n_steps):
        prop = theta + scale * prop_std[None, :] * mcmc_normals(seed, step, C, d)
        llp = ll_of_theta(prop)
        lr = (llp - ll) * inv_npts
        lu = mcmc_log_uniform(seed, step, C)
        a = (lr > 0) | ((lu > lr) if rule == 0 else (lu < lr))
        a &= ~np.isnan(lr)
        theta[a] = prop[a]
        ll[a] = llp[a]
        acc[step] = a
    return theta, ll, acc


def nproc() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1
