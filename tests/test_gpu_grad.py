"""Adjoint gradients behind torch.autograd against FP64 central finite
differences (step 1e-6), for L = 0.5 ||T_theta(x) - y||^2 with y = T_theta'(x)
for a second prior draw.

scheme="simple" (cpab_grad_theta, the midpoint scheme): differences of the
forward itself; tolerance 1e-5 relative to max|grad| (the map is piecewise
smooth: a perturbation may move a sub-step across a cell face, where the CPA
velocity is continuous but its derivative is not).

scheme="ref" (cpab_grad_theta_ref, calc_T): a step switches between the
closed-form step and the sub-step fallback where its end point crosses a
cell face, and there the map jumps (by the sub-steps' discretisation error),
so plain differences are meaningless wherever a perturbation flips a branch.
The check records the forward's branches (kept / fallback per step and the
cell of every sub-step) with a numpy restatement of calc_T's FP64 arithmetic
and the oracle's exact cell lookup, and differentiates that frozen-branch
map, which is smooth; tolerance 1e-6 relative to max|grad|."""
import numpy as np
import pytest
import torch

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.autograd import transform
from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _setup(dim, nCs, tess, n, seed, ls=0.1, var=1.0):
    sp = CpaSpace([0.0] * dim, [1.0] * dim, nCs, tess=tess, device=DEV)
    rng = np.random.default_rng(seed)
    pr = Prior.create(sp.geo, ls, var)
    th = torch.as_tensor(pr.sample(2, rng), device=DEV)
    x = torch.as_tensor(rng.uniform(0.05, 0.95, size=(n, dim)), device=DEV)
    return sp, th[:1].clone(), th[1:].clone(), x


def _loss(sp, theta, x, y, p):
    with torch.no_grad():
        out = transform(theta, x, sp, scheme="simple", **p)
    return 0.5 * ((out - y) ** 2).sum().item()


@pytest.mark.parametrize("dim,nCs,tess,ls,var", [(1, (20,), "II", 0.1, 1.0), (2, (4, 4), "I", 0.1, 1.0),
                                                 (3, (2, 2, 2), "I", 0.15, 0.5)])
def test_grad_vs_central_fd(dim, nCs, tess, ls, var):
    p = dict(dt=0.05, nTimeSteps=20, nStepsODEsolver=10)
    sp, th, th2, x = _setup(dim, nCs, tess, 400, 3, ls, var)
    with torch.no_grad():
        y = transform(th2, x, sp, scheme="simple", **p)
    t = th.clone().requires_grad_(True)
    out = transform(t, x, sp, scheme="simple", **p)
    loss = 0.5 * ((out - y) ** 2).sum()
    loss.backward()
    g = t.grad[0].cpu().numpy()
    h = 1e-6
    fd = np.empty_like(g)
    for j in range(sp.d):
        e = torch.zeros_like(th)
        e[0, j] = h
        fd[j] = (_loss(sp, th + e, x, y, p) - _loss(sp, th - e, x, y, p)) / (2 * h)
    err = np.abs(g - fd).max() / np.abs(fd).max()
    print(f"dim {dim}: d={sp.d} max|fd|={np.abs(fd).max():.3e} rel err {err:.2e}")
    assert err < 1e-5


def test_forward_equals_calc_T_simple_and_ck_invariance():
    p = dict(dt=0.02, nTimeSteps=12, nStepsODEsolver=30)
    sp, th, th2, x = _setup(2, (4, 4), "I", 3000, 5)
    out = transform(th, x, sp, scheme="simple", **p)
    sA, _ = sp.tables_from_theta(th, p["dt"], 1)       # the same A = B theta as the transform
    sp.update_pat(sA[0])
    ref = torch.empty_like(x)
    sp.calc_T_simple(pts=x, out=ref, **p)
    assert torch.equal(out, ref)
    grads = []
    for ck in (1, 5, 12):
        t = th.clone().requires_grad_(True)
        xx = x.clone().requires_grad_(True)
        o = transform(t, xx, sp, ck=ck, scheme="simple", **p)
        (o ** 2).sum().backward()
        grads.append((t.grad.clone(), xx.grad.clone()))
    for gt, gx in grads[1:]:
        # per-point gradients are deterministic; the per-cell sums use atomics (order may vary)
        assert torch.equal(gx, grads[0][1])
        torch.testing.assert_close(gt, grads[0][0], rtol=1e-12, atol=0)


def test_grad_wrt_points_vs_fd():
    p = dict(dt=0.05, nTimeSteps=10, nStepsODEsolver=10)
    sp, th, _, x = _setup(2, (4, 4), "I", 64, 7)
    xx = x.clone().requires_grad_(True)
    out = transform(th, xx, sp, scheme="simple", **p)
    w = torch.linspace(-1, 1, out.numel(), device=DEV, dtype=torch.float64).reshape(out.shape)
    (out * w).sum().backward()
    h = 1e-7
    for i in range(0, 64, 9):
        for k in range(2):
            e = torch.zeros_like(x)
            e[i, k] = h
            with torch.no_grad():
                fp = (transform(th, x + e, sp, scheme="simple", **p) * w).sum().item()
                fm = (transform(th, x - e, sp, scheme="simple", **p) * w).sum().item()
            assert abs(xx.grad[i, k].item() - (fp - fm) / (2 * h)) < 1e-6


def test_batched_thetas_independent():
    p = dict(dt=0.05, nTimeSteps=8, nStepsODEsolver=10)
    sp, th, th2, x = _setup(2, (4, 4), "I", 500, 9)
    both = torch.cat([th, th2]).clone().requires_grad_(True)
    xx = torch.cat([x, x])
    (transform(both, xx, sp, scheme="simple", **p) ** 2).sum().backward()
    for i, one in enumerate((th, th2)):
        t = one.clone().requires_grad_(True)
        (transform(t, x, sp, scheme="simple", **p) ** 2).sum().backward()
        torch.testing.assert_close(both.grad[i], t.grad[0], rtol=1e-12, atol=1e-12)


# ------------------------------------------------------------ reference scheme (calc_T)


def _affine(M, p):
    """exact_affine: row r = ((M[r,0] p0 + M[r,1] p1) + ...) + M[r,D], per point (M: [n, D*(D+1)])."""
    D = p.shape[1]
    out = np.empty_like(p)
    for r in range(D):
        acc = M[:, r * (D + 1)] * p[:, 0]
        for k in range(1, D):
            acc = acc + M[:, r * (D + 1) + k] * p[:, k]
        out[:, r] = acc + M[:, r * (D + 1) + D]
    return out


def _midpoint(M, p, h):
    """exact_midpoint: pm = p + (h v)/2, p' = p + v(pm) h, both with the same cell's matrix."""
    pm = p + (h * _affine(M, p)) / 2.0
    return p + _affine(M, pm) * h


def _ref_forward(O, t, sA, Tr, x, dt, nT, nODE, branches=None):
    """calc_T in numpy for one instance; records the branches, or replays given ones."""
    p = x.copy()
    h = dt / nODE
    rec = branches is None
    if rec:
        branches = (np.zeros((nT, len(x)), bool), np.zeros((nT, len(x)), np.int64),
                    np.zeros((nT, nODE, len(x)), np.int64))
    kept, cells, sub = branches
    for s in range(nT):
        c = O.calc_cell_idx(t, p).astype(np.int64) if rec else cells[s]
        q = _affine(Tr[c], p)
        if rec:
            kept[s] = O.calc_cell_idx(t, q) == c
            cells[s] = c
        pf = p.copy()
        for k in range(nODE):
            cc = O.calc_cell_idx(t, pf).astype(np.int64) if rec else sub[s, k]
            if rec:
                sub[s, k] = cc
            pf = _midpoint(sA[cc], pf, h)
        p = np.where(kept[s][:, None], q, pf)
    return p, branches


def _tables_np(sp, theta, dt):
    ne = sp.dim * (sp.dim + 1)
    sA, Tr = sp.tables_from_theta(theta, dt, 1)
    return sA[0].cpu().numpy().reshape(-1, ne), Tr[0].cpu().numpy().reshape(-1, ne)


# (3, (4, 4, 4), "I"): 320 cells, whose gradient sums exceed the kernel's shared-memory budget and go
# straight to global memory
@pytest.mark.parametrize("dim,nCs,tess,ls,var", [(1, (20,), "II", 0.1, 1.0), (2, (4, 4), "I", 0.1, 1.0),
                                                 (2, (3, 3), "II", 0.1, 1.0), (3, (2, 2, 2), "I", 0.15, 0.5),
                                                 (3, (4, 4, 4), "I", 0.15, 0.5)])
def test_ref_grad_vs_frozen_branch_fd(oracle_mod, dim, nCs, tess, ls, var):
    O = oracle_mod
    p = dict(dt=0.05, nTimeSteps=20, nStepsODEsolver=10)
    dt, nT, nODE = p["dt"], p["nTimeSteps"], p["nStepsODEsolver"]
    sp, th, th2, x = _setup(dim, nCs, tess, 300, 11, ls, var)
    t_or = O.tess_struct(dim, sp.geo.tess_code, sp.geo.nCs, sp.incs)
    with torch.no_grad():
        y = transform(th2, x, sp, **p)
    t = th.clone().requires_grad_(True)
    xx = x.clone().requires_grad_(True)
    out = transform(t, xx, sp, **p)
    w = torch.linspace(-1, 1, out.numel(), device=DEV, dtype=torch.float64).reshape(out.shape)
    loss = 0.5 * ((out - y) ** 2).sum() + (out * w).sum()
    loss.backward()
    g = t.grad[0].cpu().numpy()
    gx = xx.grad.cpu().numpy()
    xn, yn, wn = x.cpu().numpy(), y.cpu().numpy(), w.cpu().numpy()
    # the numpy restatement reproduces the GPU forward and records its branches
    sA0, Tr0 = _tables_np(sp, th, dt)
    out_np, br = _ref_forward(O, t_or, sA0, Tr0, xn, dt, nT, nODE)
    np.testing.assert_array_equal(out_np, out.detach().cpu().numpy())
    kept_frac = br[0].mean()
    assert 0.0 < kept_frac < 1.0, kept_frac  # both branches occur

    def L(theta=None, xs=xn):
        sA, Tr = (sA0, Tr0) if theta is None else _tables_np(sp, theta, dt)
        o, _ = _ref_forward(O, t_or, sA, Tr, xs, dt, nT, nODE, br)
        return 0.5 * ((o - yn) ** 2).sum() + (o * wn).sum()

    h = 1e-6
    comps = np.arange(sp.d) if sp.d <= 80 else np.random.default_rng(0).choice(sp.d, 60, replace=False)
    fd = np.empty(len(comps))
    for m, j in enumerate(comps):
        e = torch.zeros_like(th)
        e[0, j] = h
        fd[m] = (L(th + e) - L(th - e)) / (2 * h)
    g = g[comps]
    err = np.abs(g - fd).max() / np.abs(fd).max()
    print(f"dim {dim} tess {tess}: d={sp.d} kept {kept_frac:.3f} max|fd|={np.abs(fd).max():.3e} rel err {err:.2e}")
    assert err < 1e-6
    # dLoss/dx through the same frozen branches, for a few points
    for i in range(0, 300, 37):
        for k in range(dim):
            e = np.zeros_like(xn)
            e[i, k] = h
            fdx = (L(None, xn + e) - L(None, xn - e)) / (2 * h)
            assert abs(gx[i, k] - fdx) <= 1e-6 * max(1.0, abs(fdx))


def test_ref_forward_is_calc_T_and_ck_invariance():
    p = dict(dt=0.02, nTimeSteps=12, nStepsODEsolver=30)
    sp, th, th2, x = _setup(2, (4, 4), "I", 3000, 5)
    out = transform(th, x, sp, **p)
    sA, Tr = sp.tables_from_theta(th, p["dt"], 1)
    ref = torch.empty_like(x)
    sp.calc_T_batched((sA, Tr), x, ref, scheme=_lib.SCHEME_REF, **p)
    assert torch.equal(out, ref)
    grads = []
    for ck in (1, 5, 12):
        t = th.clone().requires_grad_(True)
        xx = x.clone().requires_grad_(True)
        o = transform(t, xx, sp, ck=ck, **p)
        (o ** 2).sum().backward()
        grads.append((t.grad.clone(), xx.grad.clone()))
    for gt, gx in grads[1:]:
        # per-point gradients are deterministic; the per-cell sums use atomics (order may vary)
        assert torch.equal(gx, grads[0][1])
        torch.testing.assert_close(gt, grads[0][0], rtol=1e-12, atol=0)


def test_ref_batched_thetas_independent_and_inverse():
    p = dict(dt=0.05, nTimeSteps=8, nStepsODEsolver=10)
    sp, th, th2, x = _setup(3, (2, 2, 2), "I", 500, 9, 0.15, 0.5)
    for sign in (1, -1):
        both = torch.cat([th, th2]).clone().requires_grad_(True)
        xx = torch.cat([x, x])
        (transform(both, xx, sp, mysign=sign, **p) ** 2).sum().backward()
        for i, one in enumerate((th, th2)):
            t = one.clone().requires_grad_(True)
            (transform(t, x, sp, mysign=sign, **p) ** 2).sum().backward()
            torch.testing.assert_close(both.grad[i], t.grad[0], rtol=1e-12, atol=1e-12)


# FP32 points (scheme="ref"): the FP32 calc_T and its adjoint.  The FP32 forward differs from the FP64 one by
# ~1e-7 and may take the other branch at a step whose end point lies that close to a cell face, so its
# gradient is compared with the FP64 adjoint's: 2e-3 relative to max|grad|.
@pytest.mark.parametrize("dim,nCs,tess,ls,var", [(1, (20,), "II", 0.1, 1.0), (2, (4, 4), "I", 0.1, 1.0),
                                                 (3, (2, 2, 2), "I", 0.15, 0.5), (3, (4, 4, 4), "I", 0.15, 0.5)])
def test_ref_grad_f32_vs_f64(dim, nCs, tess, ls, var):
    p = dict(dt=0.05, nTimeSteps=20, nStepsODEsolver=10)
    sp, th, th2, x = _setup(dim, nCs, tess, 2000, 13, ls, var)
    sp32 = CpaSpace([0.0] * dim, [1.0] * dim, nCs, tess=tess, device=DEV, precision=torch.float32)
    x32 = x.float()
    x64 = x32.double()
    with torch.no_grad():
        y = transform(th2, x64, sp, **p)
    grads = {}
    for name, s_, xx0 in (("f64", sp, x64), ("f32", sp32, x32)):
        t = th.clone().requires_grad_(True)
        xx = xx0.clone().requires_grad_(True)
        out = transform(t, xx, s_, **p)
        (0.5 * ((out.double() - y) ** 2).sum()).backward()
        grads[name] = (t.grad[0].cpu().numpy(), xx.grad.double().cpu().numpy(), out.detach())
    # the FP32 forward of the adjoint is calc_T in FP32, bit for bit
    sA, Tr = sp32.tables_from_theta(th, p["dt"], 1)
    ref = torch.empty_like(x32)
    sp32.calc_T_batched((sA, Tr), x32, ref, scheme=_lib.SCHEME_REF, **p)
    assert torch.equal(grads["f32"][2], ref)
    g64, g32 = grads["f64"][0], grads["f32"][0]
    err = np.abs(g32 - g64).max() / np.abs(g64).max()
    errx = np.abs(grads["f32"][1] - grads["f64"][1]).max() / np.abs(grads["f64"][1]).max()
    print(f"dim {dim} {nCs}: d={sp.d} FP32 vs FP64 gradient rel err {err:.2e} (points {errx:.2e})")
    assert err < 2e-3 and errx < 2e-3


def test_ref_grad_f32_ck_invariance():
    p = dict(dt=0.02, nTimeSteps=12, nStepsODEsolver=30)
    sp = CpaSpace([0.0, 0.0], [1.0, 1.0], (4, 4), tess="I", device=DEV, precision=torch.float32)
    rng = np.random.default_rng(21)
    th = torch.as_tensor(Prior.create(sp.geo, 0.1, 1.0).sample(2, rng), device=DEV)
    x = torch.as_tensor(rng.uniform(0.05, 0.95, size=(2 * 1500, 2)).astype(np.float32), device=DEV)
    grads = []
    for ck in (1, 5, 12):
        t = th.clone().requires_grad_(True)
        xx = x.clone().requires_grad_(True)
        transform(t, xx, sp, ck=ck, **p).pow(2).sum().backward()
        grads.append((t.grad.clone(), xx.grad.clone()))
    for gt, gx in grads[1:]:
        assert torch.equal(gx, grads[0][1])
        torch.testing.assert_close(gt, grads[0][0], rtol=1e-6, atol=0)
