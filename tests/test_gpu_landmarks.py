"""Batched Gaussian landmark log-likelihood (cpab_landmark_ll) against the
oracle: the oracle integrates the same landmarks with the same tables (the
reference's calc_T scheme), then sums -0.5 |T(src) - dst|^2 / sigma^2.

Tolerances: transformed landmarks bit-exact in FP64 (same tables, same
scheme); log-likelihoods 1e-12 relative in FP64 (the sum order differs),
1e-6 relative in FP32 (the FP32 likelihood tolerance)."""
import numpy as np
import pytest
import torch

from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.landmarks import LandmarkLogLikelihood
from cpabdiffeo_b200.mcmc import BatchedMetropolis
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
P = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)
SIGMA = 0.05

SPACES = {
    "1d": dict(xmins=[0.0], xmaxs=[1.0], nCs=(20,), tess="II"),
    "2d_I": dict(xmins=[0.0, 0.0], xmaxs=[1.0, 1.0], nCs=(4, 4), tess="I"),
    "2d_II": dict(xmins=[0.0, 0.0], xmaxs=[1.0, 1.0], nCs=(3, 4), tess="II"),
    "3d_I": dict(xmins=[0.0] * 3, xmaxs=[1.0] * 3, nCs=(2, 2, 2), tess="I"),
}


def _space(name, precision=torch.float64):
    s = SPACES[name]
    return CpaSpace(s["xmins"], s["xmaxs"], s["nCs"], tess=s["tess"], device=DEV, precision=precision)


def _landmarks(rng, n, dim):
    src = rng.uniform(0.02, 0.98, size=(n, dim))
    src[:3] = np.round(src[:3] * 4) / 4          # a few on cell boundaries
    dst = np.clip(src + rng.normal(0, 0.05, size=src.shape), 0, 1)
    return src, dst


def _oracle(O, sp, tables, src, dst):
    """(ll [N], transformed [N, n, dim]) from the oracle with the GPU's tables."""
    sA, Tr = (x.cpu().numpy() for x in tables)
    t = O.tess_struct(sp.dim, sp.geo.tess_code, sp.geo.nCs, sp.geo.incs)
    N = sA.shape[0]
    outs, lls = [], []
    for n in range(N):
        s_n = src if src.ndim == 2 else src[n]
        d_n = dst if dst.ndim == 2 else dst[n]
        out, _ = O.calc_T(t, Tr[n], sA[n], s_n, P["dt"], P["nTimeSteps"], P["nStepsODEsolver"])
        if sp.dim == 1:
            out = O.clamp_1d(out)
        outs.append(out)
        lls.append(float(np.sum(-0.5 * ((out - d_n) ** 2).sum(axis=1) / SIGMA ** 2)))
    return np.array(lls), np.stack(outs)


@pytest.mark.parametrize("name", list(SPACES))
def test_landmark_ll_matches_oracle_f64(oracle_mod, name):
    sp = _space(name)
    rng = np.random.default_rng(3)
    src, dst = _landmarks(rng, 57, sp.dim)
    theta = torch.as_tensor(Prior.create(sp.geo, 0.2, 1.0).sample(6, rng), device=DEV)
    ll_fn = LandmarkLogLikelihood(sp, src, dst, SIGMA, P)
    tables = sp.tables_from_theta(theta, P["dt"], 1)
    tr = torch.empty((6, 57, sp.dim), dtype=torch.float64, device=DEV)
    ll = ll_fn.batch_tables(tables, transformed=tr).cpu().numpy()
    ll_o, tr_o = _oracle(oracle_mod, sp, tables, src, dst)
    assert np.array_equal(tr.cpu().numpy(), tr_o)
    np.testing.assert_allclose(ll, ll_o, rtol=1e-12)


@pytest.mark.parametrize("name", ["2d_I", "3d_I"])
def test_landmark_ll_f32_within_1e6(oracle_mod, name):
    sp = _space(name, torch.float32)
    rng = np.random.default_rng(4)
    src, dst = _landmarks(rng, 200, sp.dim)
    theta = torch.as_tensor(Prior.create(sp.geo, 0.2, 1.0).sample(4, rng), device=DEV)
    ll_fn = LandmarkLogLikelihood(sp, src, dst, SIGMA, P)
    tables = sp.tables_from_theta(theta, P["dt"], 1)
    ll = ll_fn.batch_tables(tables).cpu().numpy()
    ll_o, _ = _oracle(oracle_mod, sp, tables, src, dst)
    np.testing.assert_allclose(ll, ll_o, rtol=1e-6)


def test_landmark_ll_per_theta_sets_and_batch_invariance():
    sp = _space("2d_I")
    rng = np.random.default_rng(5)
    N, n = 5, 3000                                  # more than one tile per instance
    sets = [_landmarks(rng, n, 2) for _ in range(N)]
    src = np.stack([s for s, _ in sets])
    dst = np.stack([d for _, d in sets])
    theta = torch.as_tensor(Prior.create(sp.geo, 0.2, 1.0).sample(N, rng), device=DEV)
    batched = LandmarkLogLikelihood(sp, src, dst, SIGMA, P).batch(theta)
    for k in range(N):
        alone = LandmarkLogLikelihood(sp, src[k], dst[k], SIGMA, P).batch(theta[k:k + 1])
        assert torch.equal(alone[0], batched[k])


def test_call_matches_reference_convention():
    """2D __call__ is the mean over landmarks, 1D __call__ the sum."""
    rng = np.random.default_rng(6)
    for name in ("1d", "2d_I"):
        sp = _space(name)
        src, dst = _landmarks(rng, 40, sp.dim)
        f = LandmarkLogLikelihood(sp, src, dst, SIGMA, P)
        th = Prior.create(sp.geo, 0.2, 1.0).sample(1, rng)[0]
        s = f.batch(torch.as_tensor(th, device=DEV).reshape(1, -1))[0].item()
        assert f(th) == pytest.approx(s if sp.dim == 1 else s / 40, rel=0, abs=0)


def test_mcmc_with_landmarks_improves_fit():
    """BatchedMetropolis drives landmark chains (calc_T_fwd tables) toward the target."""
    sp = _space("2d_I")
    rng = np.random.default_rng(7)
    prior = Prior.create(sp.geo, 0.2, 1.0)
    src, _ = _landmarks(rng, 60, 2)
    th_star = torch.as_tensor(prior.sample(1, rng), device=DEV)
    tr = torch.empty((1, 60, 2), dtype=torch.float64, device=DEV)
    LandmarkLogLikelihood(sp, src, src, SIGMA, P).batch(th_star, transformed=tr)
    dst = tr[0].cpu().numpy()
    C = 16
    ll_fn = LandmarkLogLikelihood(sp, src, dst, SIGMA, P, n_theta=C)
    mh = BatchedMetropolis(ll_fn, torch.zeros((C, sp.d), device=DEV), np.sqrt(np.diag(prior.cov_cpa)),
                           scale=0.05, seed=9)
    ll0 = mh.ll.clone()
    mh.run(200, graph_steps=50)
    torch.cuda.synchronize()
    assert (mh.ll > ll0).float().mean() > 0.9
    # the chains' current ll is the likelihood of their current theta
    torch.testing.assert_close(mh.ll, ll_fn.batch(mh.theta), rtol=0, atol=0)
