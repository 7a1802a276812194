"""Golden fixtures from the reference's own Python code, run here.

The reference's Python modules (Python 2, importing the absent `of`) are
loaded unmodified from the checkout through tests/golden/py2ref.py, which
applies only mechanical Python 2 -> 3 rewrites in memory.  This script feeds
them seeded inputs and stores inputs and outputs as .npz fixtures:

  pyref/closedform_1d.npz
                     cpab/cpa1d/calcs/ClosedFormInt.py (calc_phi :64-165,
                     find_crossing_time :193-256, calc_affine_phi :171-192):
                     the exact 1D flow at t = 1 of prior draws, forward (A)
                     and inverse (-A), on uniform points, every vertex and
                     its 1e-17 / 1e-16 / 1e-12 neighbours, the domain ends
                     and points outside.  status: 0 ok, 1 the reference
                     raised ValueError after nC crossings (:155-160),
                     2 any other exception.
  pyref/setup_<space>.npz
                     the reference's space construction:
                     cells (Tessellation.cells_verts_homo_coo), the
                     constraint matrix L (continuity + zero velocity across
                     the boundary) and B = null(L) (cpab/cpaNd/utils/_null.py),
                     stored as d and B's projector applied to a seeded sketch
                     (B itself is defined up to rotation); and the prior's
                     Sigma_PA (cpab/distributions/create_joint_algebra_cov.py)
                     for the cells, stored as the per-entry diagonals of its
                     cell blocks (every other entry is zero, checked here).

  pyref/metropolis.npz
                     cpab/cpaNd/inference/Metropolis.py + Proposal.py, one
                     chain per image pair, its random draws replaced by the
                     library's Philox streams (see make_metropolis).
  pyref/multiscale.npz
                     cpab/cpaNd/_Multiscale.py propogate_Avees_coarser2fine.

Run where the reference checkout exists (CPAB_REF_ROOT or the default mount):
    python tests/golden/make_golden_py_ref.py [closedform] [setup] [metropolis] [multiscale]
"""
from __future__ import annotations

import sys
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "pyref"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

from py2ref import Py2Loader  # noqa: E402

from cpabdiffeo_b200.space import Prior, build_space  # noqa: E402

# spaces whose construction is pinned: name -> (dim, nCs, tess)
SPACES = {
    "d1_nc100": (1, (100,), "II"),
    "d1_nc20": (1, (20,), "II"),
    "d2_tessI_4x4": (2, (4, 4), "I"),
    "d2_tessII_4x4": (2, (4, 4), "II"),
    "d2_tessI_2x3": (2, (2, 3), "I"),
    "d3_tessI_2x2x2": (3, (2, 2, 2), "I"),
    "d3_tessII_2x2x2": (3, (2, 2, 2), "II"),
    "d3_tessI_4x4x4": (3, (4, 4, 4), "I"),
}
# prior parameters per space: length scale (domain units), variance; the
# per-dimension left/right scales are the TransformWrapper defaults
PRIOR = {1: (0.1, 1.0), 2: (0.1, 1.0), 3: (0.15, 0.5)}
SKETCH_COLS = 8


# ----------------------------------------------------------------------------- ClosedFormInt


def _tw_standin(nC: int, A: np.ndarray):
    """The attributes ClosedFormInt reads from a TransformWrapper
    (ClosedFormInt.py:14-20): ms.L_cpa_space[0].{nC, local_stuff.vert_tess, pat.As_sq_mats}."""
    x_tess = np.linspace(0.0, 1.0, nC + 1)
    As_sq = np.zeros((nC, 2, 2))
    As_sq[:, 0, :] = A
    space = types.SimpleNamespace(nC=nC, local_stuff=types.SimpleNamespace(vert_tess=x_tess[:, None].copy()),
                                  pat=types.SimpleNamespace(As_sq_mats=As_sq))
    return types.SimpleNamespace(ms=types.SimpleNamespace(L_cpa_space=[space])), x_tess


def vertex_velocities(A: np.ndarray, x_tess: np.ndarray) -> np.ndarray:
    """velTess: the velocity at each vertex, from the cell to its right
    (the last vertex from the last cell); continuous fields agree with the
    cell to the left up to rounding."""
    nC = A.shape[0]
    c = np.minimum(np.arange(nC + 1), nC - 1)
    return (A[c, 0] * x_tess + A[c, 1])[:, None]


def closed_form_points(nC: int, rng) -> np.ndarray:
    v = np.linspace(0.0, 1.0, nC + 1)
    pts = [rng.uniform(0, 1, 240), v, (np.arange(nC) + 0.5) / nC]
    for eps in (1e-17, 1e-16, 1e-12):
        pts += [v[1:-1] - eps, v[1:-1] + eps]
    pts.append(np.array([0.0, -0.0, 1.0, 1e-300, 1 - 1e-16, 1e-16, -1e-12, 1 + 1e-12, -0.3, 1.4]))
    return np.concatenate(pts)


def _raised_at_cap(ex: BaseException) -> bool:
    """True when calc_phi gave up after nC crossings: the exception comes from
    its `raise ValueError(x_old, x_new, ..., v, ...)` statement (evaluating
    its arguments may itself raise UnboundLocalError for `v`, as in Python 2)."""
    tb = ex.__traceback__
    while tb.tb_next is not None:
        tb = tb.tb_next
    f = tb.tb_frame
    return f.f_code.co_name == "calc_phi" and CAP_RAISE_LINES[0] <= tb.tb_lineno <= CAP_RAISE_LINES[1]


# the statement in ClosedFormInt.calc_phi that raises after nC crossings
CAP_RAISE_LINES = (158, 160)


def make_closedform(L: Py2Loader) -> None:
    CFI = L.load("cpab/cpa1d/calcs/ClosedFormInt.py").ClosedFormInt
    cases = [(100, 10, 1.0), (20, 3, 1.0), (5, 3, 6.0)]   # nC, theta draws, prior std multiplier
    rng = np.random.default_rng(11)
    rec = {k: [] for k in ("nC", "A", "x", "out", "status", "case")}
    t0 = time.time()
    for ci, (nC, n_theta, mult) in enumerate(cases):
        geo = build_space(1, (nC,), "II")
        prior = Prior.create(geo, *PRIOR[1])
        theta = prior.sample(n_theta, rng) * mult
        for i in range(n_theta):
            A0 = (geo.B @ theta[i]).reshape(nC, 2)
            x = closed_form_points(nC, rng)
            for sign in (1, -1):
                A = sign * A0
                tw, x_tess = _tw_standin(nC, A)
                cfi = CFI(tw)
                vel = vertex_velocities(A, x_tess)
                out = np.full(x.size, np.nan)
                status = np.zeros(x.size, dtype=np.int8)
                for k, xk in enumerate(x):
                    try:
                        out[k] = cfi.calc_phi(float(xk), velTess=vel, t=1.0)
                    except Exception as ex:  # noqa: BLE001 -- recorded, never silently dropped
                        status[k] = 1 if _raised_at_cap(ex) else 2
                rec["nC"].append(nC)
                rec["A"].append(A.ravel())
                rec["x"].append(x)
                rec["out"].append(out)
                rec["status"].append(status)
                rec["case"].append(ci)
    lens = np.array([a.size for a in rec["x"]])
    np.savez_compressed(OUT / "closedform_1d.npz",
                        nC=np.array(rec["nC"]), case=np.array(rec["case"]),
                        A_offsets=np.concatenate([[0], np.cumsum([a.size for a in rec["A"]])]),
                        A=np.concatenate(rec["A"]),
                        offsets=np.concatenate([[0], np.cumsum(lens)]),
                        x=np.concatenate(rec["x"]), out=np.concatenate(rec["out"]),
                        status=np.concatenate(rec["status"]), t=np.array(1.0))
    st = np.concatenate(rec["status"])
    print(f"closedform_1d: {len(rec['nC'])} flows, {lens.sum()} points, "
          f"{(st == 1).sum()} capped, {(st == 2).sum()} other, {time.time() - t0:.1f} s")


# ----------------------------------------------------------------------------- space construction


def reference_space(L: Py2Loader, dim: int, nCs, tess: str):
    """cells, L and B as the reference's CpaSpace builds them
    (cpab/cpa1d/CpaSpace.py:57-107, cpab/cpa2d/CpaSpace.py:79-172,
    cpab/cpa3d/CpaSpace.py) with zero velocity across every boundary face,
    valid_outside=False, no volume preservation."""
    XMINS, XMAXS = [0.0] * dim, [1.0] * dim
    null = L.load("cpab/cpaNd/utils/_null.py").null
    if dim == 1:
        T = L.load("cpab/cpa1d/Tessellation.py").Tessellation(nCx=nCs[0], XMINS=XMINS, XMAXS=XMAXS)
        verts1, H, nEdges, nConstraints = T.create_verts_and_H()
        cc = L.load("cpab/cpa1d/utils/constraints/_create_cont_constraint_mat.py").create_cont_constraint_mat
        Lm = cc(H, verts1, nEdges, nConstraints, T.nC, dim_domain=1)
    elif dim == 2:
        nC = nCs[0] * nCs[1] * (4 if tess == "I" else 1)
        T = L.load("cpab/cpa2d/Tessellation.py").Tessellation(nCs[0], nCs[1], nC, XMINS, XMAXS, tess=tess)
        verts1, verts2, H, nEdges, nConstraints = T.create_verts_and_H(dim_range=2, valid_outside=False)
        cc = L.load("cpab/cpa2d/utils/constraints/_create_cont_constraint_mat.py").create_cont_constraint_mat
        Lm = cc(H, verts1, verts2, nEdges, nConstraints, nC, dim_domain=2, dim_range=2)
    else:
        nC = nCs[0] * nCs[1] * nCs[2] * (5 if tess == "I" else 1)
        T = L.load("cpab/cpa3d/Tessellation.py").Tessellation(nCs[0], nCs[1], nCs[2], nC, XMINS, XMAXS, tess=tess)
        v1, v2, v3, v4, H, nSides, nConstraints = T.create_verts_and_H(dim_range=3, valid_outside=False)
        cc = L.load("cpab/cpa3d/utils/constraints/_create_cont_constraint_mat.py").create_cont_constraint_mat
        Lm = cc(H, v1, v2, v3, v4, nSides, nConstraints, nC, dim_domain=3, dim_range=3, tess=tess)
    Lb = T.create_constraint_mat_bdry(zero_v_across_bdry=[True] * dim)
    Lm = np.vstack([Lm, Lb])
    B = null(Lm)
    return T, np.asarray(T.cells_verts_homo_coo, dtype=np.float64), Lm, B


def make_setup(L: Py2Loader, names=None) -> None:
    cov_fn = L.load("cpab/distributions/create_joint_algebra_cov.py").create_joint_algebra_cov
    for name, (dim, nCs, tess) in SPACES.items():
        if names and name not in names:
            continue
        t0 = time.time()
        T, cells, Lm, B = reference_space(L, dim, nCs, tess)
        D, d = B.shape
        sk = np.random.default_rng(123).standard_normal((D, SKETCH_COLS))
        proj_sketch = B @ (B.T @ sk)
        # the prior's Sigma_PA for these cells (the pa_space attributes the function reads)
        geo = build_space(dim, nCs, tess)
        ls, var = PRIOR[dim]
        centers = cells.mean(axis=1)
        d0 = np.linalg.norm(centers[0] - centers[1])
        left = 1.0 if dim == 1 else 0.01
        pas = types.SimpleNamespace(tessellation=T, lengthAvee=dim * (dim + 1), dim_domain=dim, dim_range=dim,
                                    XMINS=np.zeros(dim), XMAXS=np.ones(dim), nC=cells.shape[0])
        cov = cov_fn(pas, scale_spatial=ls / d0, scale_value=np.sqrt(var), left_blk_rel_scale=left,
                     right_vec_scale=1.0)
        nC, ne = cells.shape[0], dim * (dim + 1)
        blk = cov.reshape(nC, ne, nC, ne)
        diag = np.einsum("ikjk->ijk", blk)                 # [nC, nC, ne]: block (i, j) diagonal
        off = blk.copy()
        for k in range(ne):
            off[:, k, :, k] = 0
        if np.abs(off).max() != 0:
            raise AssertionError(f"{name}: Sigma_PA has entries off the block diagonals")
        np.savez_compressed(OUT / f"setup_{name}.npz", dim=dim, nCs=np.array(nCs), tess=np.array(tess),
                            cells=cells, n_constraints=np.array(Lm.shape[0]), rank_L=np.array(np.linalg.matrix_rank(Lm)),
                            d=np.array(d), sketch_seed=np.array(123), proj_sketch=proj_sketch,
                            prior_length_scale=np.array(ls), prior_variance=np.array(var),
                            prior_left_blk_rel_scale=np.array(left), prior_scale_spatial=np.array(ls / d0),
                            sigma_pa_block_diag=diag)
        print(f"setup_{name}: nC={nC} D={D} d={d} L={Lm.shape} ({time.time() - t0:.1f} s); "
              f"ours d={geo.d}")


# ----------------------------------------------------------------------------- Metropolis


MH = dict(H=24, W=24, chains=3, steps=14, seed=77, scale=0.05, sigma=0.05, dt=0.02, nT=50, nODE=100)


def mh_problem():
    """A small registration problem: 2D type I 4x4, three image pairs."""
    from scipy.ndimage import gaussian_filter

    from oracle import oracle as O
    geo = build_space(2, (4, 4), "I")
    prior = Prior.create(geo, *PRIOR[2])
    rng = np.random.default_rng(101)
    C, H, W = MH["chains"], MH["H"], MH["W"]
    src = np.stack([gaussian_filter(rng.uniform(0, 1, (H, W)), 2.0).astype(np.float32) for _ in range(C)])
    dst = np.stack([np.roll(src[c], 1, axis=1) + rng.normal(0, 0.02, (H, W)).astype(np.float32)
                    for c in range(C)]).astype(np.float32)
    t = O.tess_struct(2, 1, (4, 4), geo.incs)

    def ll_one(theta, c):
        sA, Tr = O.expm_cells(2, geo.B @ theta, MH["dt"], -1)
        v, _ = O.register_ll(t, Tr, sA, src[c], dst[c], MH["sigma"], MH["dt"], MH["nT"], MH["nODE"])
        return v
    return geo, prior, src, dst, ll_one


class _LLStandIn:
    """What Metropolis reads from its likelihood: a call theta -> ll, .level
    and ._ll_func.nPts (Metropolis.py:19, :31-32, :58-59)."""

    def __init__(self, fn, n_pts):
        self.fn = fn
        self.level = 0
        self._ll_func = types.SimpleNamespace(nPts=n_pts)

    def __call__(self, theta):
        return self.fn(theta)


def make_metropolis(L: Py2Loader) -> None:
    """cpab/cpaNd/inference/Metropolis.py (set_theta :25-40, step :41-85,
    accept :87-99) with cpab/cpaNd/inference/Proposal.py (:29-64, the
    diagonal-covariance random walk), one chain per image pair.  The two
    random sources are replaced by the library's Philox streams: the
    proposal's multivariate-normal draw (Proposal.py:61-64 passes
    cov = scale^2 diag(Sigma_CPA)) returns mean + sqrt(diag(cov)) z with z
    the chain's normals at that step, and np.random.rand returns the chain's
    uniform at that step -- so the chain can be compared draw for draw."""
    from oracle import oracle as O
    met = L.load("cpab/cpaNd/inference/Metropolis.py")
    prop_mod = L.load("cpab/cpaNd/inference/Proposal.py")
    geo, prior, src, dst, ll_one = mh_problem()
    C, d, n_steps, seed = MH["chains"], geo.d, MH["steps"], MH["seed"]
    key = (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    thetas = np.zeros((n_steps + 1, C, d))
    lls = np.zeros((n_steps + 1, C))
    acc = np.zeros((n_steps, C), dtype=bool)
    for c in range(C):
        state = {"step": 0}

        def draw(mean, cov, c=c):
            z = O.mcmc_normals(seed, state["step"], C, d)[c]
            return mean + np.sqrt(np.diag(cov)) * z

        def rand(c=c):
            ch = np.array([c])
            ctr = np.stack([ch, np.full_like(ch, state["step"] & 0xFFFFFFFF),
                            np.full_like(ch, ((state["step"] >> 32) << 8) | 1), np.zeros_like(ch)], -1)
            r = O.philox4x32_10(ctr.astype(np.uint64), key)
            return float(O._u53(r[..., 0], r[..., 1])[0])

        prop_mod.draw_from_mvnormal = draw
        met.np = types.SimpleNamespace(**{k: getattr(np, k) for k in ("log", "float", "zeros_like", "copyto")},
                                       random=types.SimpleNamespace(rand=rand))
        ll_func = _LLStandIn(lambda th, c=c: ll_one(th, c), MH["H"] * MH["W"])
        covs = types.SimpleNamespace(cpa_cov=prior.cov_cpa)
        proposal = prop_mod.Proposal(ms=types.SimpleNamespace(L_cpa_space=[types.SimpleNamespace()]),
                                     msp=types.SimpleNamespace(L_cpa_space_covs=[covs]), level=0, scale=MH["scale"])
        mh = met.Metropolis(ll_func, proposal)
        mh.set_theta(np.zeros(d))
        thetas[0, c] = mh.theta_current
        lls[0, c] = mh.ll_current
        for k in range(n_steps):
            state["step"] = k
            before = mh.nAccepted
            mh.step()
            acc[k, c] = mh.nAccepted > before
            thetas[k + 1, c] = mh.theta_current
            lls[k + 1, c] = mh.ll_current
    np.savez_compressed(OUT / "metropolis.npz", src=src, dst=dst, theta=thetas, ll_ave=lls, accepted=acc,
                        prop_std=np.sqrt(np.diag(prior.cov_cpa)),
                        **{k: np.array(v) for k, v in MH.items()})
    print(f"metropolis: {C} chains x {n_steps} steps, accepted {acc.sum()}")


# ----------------------------------------------------------------------------- multiscale


MS_CASES = [("d1", 1, (4,), "II"), ("d2_II", 2, (2, 2), "II"), ("d2_I", 2, (2, 2), "I"), ("d3_II", 3, (2, 2, 2), "II")]


def make_multiscale(L: Py2Loader) -> None:
    """cpab/cpaNd/_Multiscale.py propogate_Avees_coarser2fine (:166-292):
    every fine cell's affine map from the coarse level (one level up, twice
    the cells per axis), on seeded random coarse matrices."""
    L.stubs["_CpaSpace"] = types.SimpleNamespace(my_dtype=np.float64)
    ms_mod = L.load("cpab/cpaNd/_Multiscale.py")
    rng = np.random.default_rng(202)
    out = {}
    for name, dim, base, tess in MS_CASES:
        ne = dim * (dim + 1)
        per = {("I", 2): 4, ("I", 3): 5}.get((tess, dim), 1)

        def sp(nCs):
            n = int(np.prod(nCs)) * per
            t = types.SimpleNamespace(nCx=nCs[0], nCy=nCs[1] if dim > 1 else 1, nCz=nCs[2] if dim > 2 else 1)
            return types.SimpleNamespace(D=n * ne, tess=tess, tessellation=t)
        coarse, fine = sp(base), sp(tuple(2 * b for b in base))
        selfstub = types.SimpleNamespace(lengthAvee=ne, dim_domain=dim, L_cpa_space=[coarse, fine])
        Ac = rng.standard_normal(coarse.D)
        Af = np.zeros(fine.D)
        ms_mod.Multiscale.propogate_Avees_coarser2fine(selfstub, Ac, Af)
        out[f"{name}_coarse"] = Ac
        out[f"{name}_fine"] = Af
    np.savez_compressed(OUT / "multiscale.npz", **out)
    print("multiscale:", ", ".join(c[0] for c in MS_CASES))


def main(argv) -> None:
    L = Py2Loader()
    what = set(argv[1:]) or {"closedform", "setup", "metropolis", "multiscale"}
    if "closedform" in what:
        make_closedform(L)
    if "setup" in what:
        make_setup(L)
    if "metropolis" in what:
        make_metropolis(L)
    if "multiscale" in what:
        make_multiscale(L)


if __name__ == "__main__":
    main(sys.argv)
