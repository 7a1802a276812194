"""Multiscale (coarse-to-fine) spaces and batched registration on the GPU."""
import numpy as np
import pytest
import torch
from scipy.ndimage import gaussian_filter

from cpabdiffeo_b200.multiscale import Multiscale, MultiscaleRegister, parent_cells
from cpabdiffeo_b200.registration import GaussianLogLikelihood
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
P = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)


@pytest.mark.parametrize("base,tess", [((2, 2), "I"), ((2, 3), "II")])
def test_propagation_matches_host_and_keeps_the_velocity(base, tess):
    ms = Multiscale([0.0, 0.0], [1.0, 1.0], base, 3, tess=tess, device=DEV)
    rng = np.random.default_rng(0)
    sc, sf = ms.L_cpa_space[0], ms.L_cpa_space[1]
    th = torch.as_tensor(rng.normal(size=(4, sc.d)), device=DEV)
    th_f = ms.propagate_theta_coarse2fine(th, 0)
    par = parent_cells(sc.geo, sf.geo)
    want = (sc.geo.B @ th.cpu().numpy().T).T.reshape(4, sc.nC, -1)[:, par].reshape(4, -1) @ sf.geo.B
    np.testing.assert_allclose(th_f.cpu().numpy(), want, rtol=1e-12, atol=1e-12)
    # the velocity field is unchanged (calc_v on both levels)
    pts = torch.as_tensor(rng.uniform(0.01, 0.99, size=(2000, 2)), device=DEV)
    for n in range(4):
        vc, vf = torch.empty_like(pts), torch.empty_like(pts)
        sc.update_pat(sc.B @ th[n])
        sc.calc_v(pts=pts, out=vc)
        sf.update_pat(sf.B @ th_f[n])
        sf.calc_v(pts=pts, out=vf)
        torch.testing.assert_close(vf, vc, rtol=0, atol=1e-10)
    # two levels at once: coarse -> middle -> fine
    th_ff = ms.propagate_theta_coarse2fine(th_f, 1)
    assert th_ff.shape == (4, ms.L_cpa_space[2].d)


def test_multiscale_register_improves_the_fit():
    C, H = 8, 48
    ms = Multiscale([0.0, 0.0], [1.0, 1.0], (2, 2), 2, tess="I", device=DEV, precision=torch.float32)
    rng = np.random.default_rng(1)
    fine = ms.L_cpa_space[1]
    src = torch.as_tensor(np.stack([gaussian_filter(rng.uniform(0, 1, (H, H)).astype(np.float32), 3.0)
                                    for _ in range(C)]), device=DEV)
    th_star = torch.as_tensor(Prior.create(fine.geo, 0.2, 1.0).sample(C, rng), device=DEV)
    warped = torch.empty_like(src)
    GaussianLogLikelihood(fine, src, src, 0.05, P).batch(th_star, warped=warped)
    dst = warped + 0.01 * torch.randn(warped.shape, generator=torch.Generator(DEV).manual_seed(0), device=DEV)
    reg = MultiscaleRegister(ms, src, dst, 0.05, P, proposal_scale=0.05, length_scale=0.2, seed=3)
    theta = reg.fit([150, 150], graph_steps=50)
    assert theta.shape == (C, fine.d)
    r0, r1 = reg.records
    # the propagated start of level 1 is as good as the end of level 0 (same field), and level 1 improves it
    torch.testing.assert_close(r1["ll_start"], r0["ll_end"], rtol=1e-4, atol=0)
    assert (r1["ll_end"] > r0["ll_start"]).float().mean() >= 0.9
