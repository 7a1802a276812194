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
