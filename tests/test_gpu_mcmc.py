"""Batched Metropolis on the GPU against the CPU oracle with the same random
stream (Philox4x32-10): identical accept decisions, final theta within 1e-12,
and a captured CUDA graph replay identical to eager steps."""
import numpy as np
import pytest
import torch
from scipy.ndimage import gaussian_filter

from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.mcmc import BatchedMetropolis
from cpabdiffeo_b200.registration import GaussianLogLikelihood
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
P = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)


def _problem(C=3, H=32, W=32, seed=11):
    sp = CpaSpace([0.0, 0.0], [1.0, 1.0], (4, 4), tess="I", device=DEV, precision=torch.float64)
    rng = np.random.default_rng(seed)
    prior = Prior.create(sp.geo, 0.1, 1.0)
    src = np.stack([gaussian_filter(rng.uniform(0, 1, (H, W)).astype(np.float32), 3.0) for _ in range(C)])
    # dst = src warped by a prior draw (through the GPU likelihood's warped output) plus noise
    theta_star = prior.sample(C, rng)
    warped = torch.empty((C, H, W), dtype=torch.float32, device=DEV)
    tmp = GaussianLogLikelihood(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(src, device=DEV), 0.05, P)
    tmp.batch(torch.as_tensor(theta_star, device=DEV), warped=warped)
    dst = warped.cpu().numpy() + rng.normal(0, 0.02, size=(C, H, W)).astype(np.float32)
    prop_std = np.sqrt(np.diag(prior.cov_cpa))
    return sp, src, dst, prop_std


def _oracle_ll_fn(O, sp, src, dst):
    t = O.tess_struct(2, 1, (4, 4), sp.incs)

    def f(theta):
        out = np.empty(theta.shape[0])
        for c in range(theta.shape[0]):
            sA, Tr = O.expm_cells(2, sp.B_host @ theta[c], P["dt"], -1)
            out[c], _ = O.register_ll(t, Tr, sA, src[c], dst[c], 0.05, P["dt"], P["nTimeSteps"],
                                      P["nStepsODEsolver"])
        return out
    return f


@pytest.mark.parametrize("rule,rule_id", [("reference", 0), ("standard", 1)])
def test_mcmc_matches_oracle(oracle_mod, rule, rule_id):
    O = oracle_mod
    sp, src, dst, prop_std = _problem()
    C, n_steps, seed = src.shape[0], 12, 1234
    ll = GaussianLogLikelihood(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.05, P)
    theta0 = np.zeros((C, sp.d))
    mh = BatchedMetropolis(ll, torch.as_tensor(theta0, device=DEV), prop_std, scale=0.05, seed=seed, rule=rule)
    accepted = []
    for _ in range(n_steps):
        before = mh.n_accepted.clone()
        mh.run(1)
        accepted.append((mh.n_accepted - before).cpu().numpy().astype(bool))
    th_o, ll_o, acc_o = O.mcmc_run(sp.B_host, _oracle_ll_fn(O, sp, src, dst), theta0, prop_std, 0.05, seed, n_steps,
                                   1.0 / (32 * 32), rule=rule_id)
    np.testing.assert_array_equal(np.asarray(accepted), acc_o)
    np.testing.assert_allclose(mh.theta.cpu().numpy(), th_o, rtol=0, atol=1e-12)
    np.testing.assert_allclose(mh.ll.cpu().numpy(), ll_o, rtol=1e-10)
    assert int(mh.step.item()) == n_steps


def test_mcmc_graph_replay_equals_eager():
    sp, src, dst, prop_std = _problem(C=4, H=24, W=28, seed=12)
    C = src.shape[0]
    ll = GaussianLogLikelihood(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.05, P)
    a = BatchedMetropolis(ll, torch.zeros((C, sp.d), device=DEV), prop_std, seed=5)
    b = BatchedMetropolis(ll, torch.zeros((C, sp.d), device=DEV), prop_std, seed=5)
    a.run(10)
    b.run(10, graph_steps=4)          # 2 replays of a 4-step graph + 2 eager steps
    torch.cuda.synchronize()
    assert torch.equal(a.theta, b.theta) and torch.equal(a.ll, b.ll)
    assert torch.equal(a.n_accepted, b.n_accepted) and int(b.step.item()) == 10


def test_local_proposal_matches_oracle_draws(oracle_mod):
    """theta' = theta + G[k] dv with the oracle's Philox stream-2 draws: dv = s z at
    an interior vertex, -E[k] theta (velocity set to 0) at a boundary vertex."""
    from cpabdiffeo_b200 import _lib
    from cpabdiffeo_b200.space import local_proposal_tables
    O = oracle_mod
    sp, src, dst, prop_std = _problem(C=64)
    ll = GaussianLogLikelihood(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.05, P)
    rng = np.random.default_rng(2)
    theta0 = Prior.create(sp.geo, 0.1, 1.0).sample(64, rng)
    mh = BatchedMetropolis(ll, torch.as_tensor(theta0, device=DEV), use_local=True, scale_local_proposal=0.3, seed=21)
    mh.step.fill_(5)
    c = sp._ctx
    c.check(c.lib.cpab_mcmc_propose_local(c.h, mh.C, mh.d, _lib.ptr(mh.theta), mh.local_nV, _lib.ptr(mh.local_E),
                                          _lib.ptr(mh.local_G), _lib.ptr(mh.local_bdry), mh.local_s, mh.seed,
                                          _lib.ptr(mh.step), _lib.ptr(mh.theta_prop), _lib.stream_ptr()))
    tabs = local_proposal_tables(sp.geo)
    k, z = O.mcmc_local_draws(21, 5, 64, tabs.vertices.shape[0], 2)
    assert tabs.bdry[k].any() and (~tabs.bdry[k]).any()          # both kinds drawn
    want = np.empty_like(theta0)
    for ch in range(64):
        dv = -tabs.E[k[ch]] @ theta0[ch] if tabs.bdry[k[ch]] else mh.local_s * z[ch]
        want[ch] = theta0[ch] + tabs.G[k[ch]] @ dv
    np.testing.assert_allclose(mh.theta_prop.cpu().numpy(), want, rtol=0, atol=1e-12)
    # the proposal moves exactly one vertex velocity
    for ch in range(8):
        v_old = np.einsum("krd,d->kr", tabs.E, theta0[ch])
        v_new = np.einsum("krd,d->kr", tabs.E, mh.theta_prop[ch].cpu().numpy())
        moved = np.abs(v_new - v_old).max(axis=1) > 1e-12
        assert moved.sum() <= 1 and (not moved.any() or moved[k[ch]])


def test_local_proposal_chains_run_and_improve():
    sp, src, dst, prop_std = _problem(C=8)
    ll = GaussianLogLikelihood(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.05, P)
    mh = BatchedMetropolis(ll, torch.zeros((8, sp.d), device=DEV), use_local=True, scale_local_proposal=0.05,
                           seed=4)
    ll0 = mh.ll.clone()
    mh.run(60, graph_steps=20)
    torch.cuda.synchronize()
    assert (mh.ll > ll0).float().mean() >= 0.75
    torch.testing.assert_close(mh.ll, ll.batch(mh.theta), rtol=0, atol=0)


def test_mcmc_run_entry_point_equals_stepwise_chains():
    """cpab_mcmc_run (one C call for n steps) enqueues the same kernels in the
    same order as BatchedMetropolis: identical chains."""
    from cpabdiffeo_b200 import _lib
    sp, src, dst, prop_std = _problem(C=4)
    srcg, dstg = torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV)
    ll_fn = GaussianLogLikelihood(sp, srcg, dstg, 0.05, P)
    mh = BatchedMetropolis(ll_fn, torch.zeros((4, sp.d), device=DEV), prop_std, scale=0.05, seed=17)
    mh.run(12)
    c = sp._ctx
    H, W = src.shape[1:]
    theta = torch.zeros((4, sp.d), dtype=torch.float64, device=DEV)
    ll = torch.empty(4, dtype=torch.float64, device=DEV)
    step = torch.zeros(1, dtype=torch.int64, device=DEV)
    acc = torch.zeros(4, dtype=torch.int64, device=DEV)
    ws = torch.empty(int(c.lib.cpab_mcmc_run_workspace_bytes(c.h, 4, sp.d, H, W)), dtype=torch.uint8, device=DEV)
    std = torch.as_tensor(prop_std, device=DEV)
    c.check(c.lib.cpab_mcmc_run(c.h, _lib.ptr(sp.B), sp.d, 4, _lib.ptr(theta), _lib.ptr(std), 0.05,
                                _lib.ptr(srcg), _lib.ptr(dstg), H, W, 0.05, _lib.CPAB_F64, P["dt"], P["nTimeSteps"],
                                P["nStepsODEsolver"], 1.0 / (H * W), 0, 17, _lib.ptr(step), 12, _lib.ptr(ll),
                                _lib.ptr(acc), _lib.ptr(ws), ws.numel(), _lib.stream_ptr()))
    torch.cuda.synchronize()
    assert torch.equal(theta, mh.theta) and torch.equal(ll, mh.ll)
    assert torch.equal(acc, mh.n_accepted) and int(step.item()) == 12
