"""GPU parity of remap, the Gaussian SSD log-likelihood and the fused
registration likelihood against the oracle (C ABI underneath).

Tolerances: remapped images 1e-5 absolute (float32 output of a double
bilinear); log-likelihoods 1e-9 relative when the oracle integrates with the
same tables (FP64), 1e-6 relative for the FP32 integration.
"""
import numpy as np
import pytest
import torch
from scipy.ndimage import gaussian_filter

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.registration import GaussianLogLikelihood, TransformWrapper, remap, remap_ssd
from cpabdiffeo_b200.space import Prior, pixel_centers

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
UNIT = lambda H, W: (W, -0.5, H, -0.5)  # noqa: E731


def smooth_image(rng, H, W, sigma=8.0):
    img = rng.uniform(0, 1, size=(H, W)).astype(np.float32)
    return gaussian_filter(img, sigma=sigma, mode="reflect").astype(np.float32)


def test_remap_matches_oracle(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(0)
    H, W = 96, 80
    src = smooth_image(rng, H, W, 3.0)
    pts = pixel_centers(H, W) + rng.normal(0, 0.05, size=(H * W, 2))
    pts[:50] = rng.uniform(-0.3, 1.3, size=(50, 2))           # outside the image too
    pts[50] = [np.nan, 0.5]
    for dt in (torch.float64, torch.float32):
        m = torch.as_tensor(pts, dtype=dt, device=DEV)
        got = remap(m, torch.as_tensor(src, device=DEV), pixel_map=UNIT(H, W)).cpu().numpy()
        want = O.remap(m.cpu().numpy().astype(np.float64), src, *UNIT(H, W))
        assert np.abs(got - want).max() < 1e-5


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_remap_unaligned_map_same_result(dt):
    """A map that starts one element past an aligned address takes the scalar
    load path and gives the same bits as the vector path."""
    rng = np.random.default_rng(5)
    H, W = 64, 48
    src = torch.as_tensor(smooth_image(rng, H, W, 2.0), device=DEV)
    pts = pixel_centers(H, W) + rng.normal(0, 0.05, size=(H * W, 2))
    m = torch.as_tensor(pts, dtype=dt, device=DEV)
    buf = torch.empty(H * W * 2 + 1, dtype=dt, device=DEV)
    mu = buf[1:].view(H * W, 2)
    mu.copy_(m)
    assert mu.data_ptr() % (2 * mu.element_size()) != 0
    a = remap(m, src, pixel_map=UNIT(H, W))
    b = remap(mu, src, pixel_map=UNIT(H, W))
    assert torch.equal(a, b)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_remap_ssd_bulk_and_plain_paths_agree(oracle_mod, dt):
    """Aligned maps of 4 | H*W pixels take the bulk-copy kernel; a map 8 bytes
    off a 16-byte boundary and an odd-sized image take the plain kernel.  Both
    give the same bits, and the oracle's values."""
    O = oracle_mod
    rng = np.random.default_rng(11)
    # (64, 128): power-of-two scales, so float maps take the float-coordinate sampler
    for H, W in ((72, 96), (63, 65), (64, 128)):
        N = 3
        src = np.stack([smooth_image(rng, H, W, 2.0) for _ in range(N)])
        dst = np.stack([smooth_image(rng, H, W, 2.0) for _ in range(N)])
        pts = pixel_centers(H, W)[None] + rng.normal(0, 0.03, size=(N, H * W, 2))
        m = torch.as_tensor(pts, dtype=dt, device=DEV).contiguous()
        buf = torch.empty(N * H * W * 2 + 16, dtype=dt, device=DEV)
        shift = 8 // m.element_size()                       # 8 bytes
        mu = buf[shift:shift + m.numel()].view(N, H * W, 2)
        mu.copy_(m)
        s_t, d_t = torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV)
        wa, wb = torch.empty_like(s_t), torch.empty_like(s_t)
        la = remap_ssd(m, s_t, d_t, 0.1, pixel_map=UNIT(H, W), warped=wa)
        lb = remap_ssd(mu, s_t, d_t, 0.1, pixel_map=UNIT(H, W), warped=wb)
        assert torch.equal(la, lb) and torch.equal(wa, wb)
        for n in range(N):
            mp = pts[n] if dt == torch.float64 else pts[n].astype(np.float32).astype(np.float64)
            ll, warped = O.remap_ssd(mp, src[n], dst[n], 0.1, *UNIT(H, W))
            assert abs(la[n].item() - ll) <= 1e-6 * abs(ll)
            assert np.abs(wa[n].cpu().numpy() - warped).max() < 1e-5


def test_remap_identity_pixel_units():
    rng = np.random.default_rng(1)
    H, W = 33, 47
    src = smooth_image(rng, H, W)
    tw = TransformWrapper(H, W, base=(2, 2), device=DEV)
    out = torch.zeros((H, W), dtype=torch.float32, device=DEV)
    tw.remap_fwd(tw.pts_src_dense, torch.as_tensor(src, device=DEV), out)
    np.testing.assert_array_equal(out.cpu().numpy(), src)


def test_remap_ssd_matches_oracle(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(2)
    N, H, W = 3, 64, 72
    src = np.stack([smooth_image(rng, H, W) for _ in range(N)])
    dst = np.stack([smooth_image(rng, H, W) for _ in range(N)])
    maps = np.stack([pixel_centers(H, W) + rng.normal(0, 0.02, size=(H * W, 2)) for _ in range(N)])
    m = torch.as_tensor(maps, device=DEV)
    warped = torch.empty((N, H, W), dtype=torch.float32, device=DEV)
    ll = remap_ssd(m, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.05,
                   pixel_map=UNIT(H, W), warped=warped).cpu().numpy()
    for n in range(N):
        ll_o, w_o = O.remap_ssd(maps[n], src[n], dst[n], 0.05, *UNIT(H, W))
        assert abs(ll[n] - ll_o) <= 1e-9 * abs(ll_o)
        assert np.abs(warped[n].cpu().numpy() - w_o).max() < 1e-5


def _register_setup(N, H, W, seed, precision=torch.float64):
    sp = CpaSpace([0.0, 0.0], [1.0, 1.0], (4, 4), tess="I", device=DEV, precision=precision)
    rng = np.random.default_rng(seed)
    prior = Prior.create(sp.geo, 0.1, 1.0)
    theta = prior.sample(N, rng)
    src = np.stack([smooth_image(rng, H, W) for _ in range(N)])
    dst = np.stack([smooth_image(rng, H, W) for _ in range(N)])
    return sp, theta, src, dst


@pytest.mark.parametrize("precision,rtol", [(torch.float64, 1e-9), (torch.float32, 1e-6)])
def test_register_ll_matches_oracle(oracle_mod, precision, rtol):
    O = oracle_mod
    N, H, W = 3, 64, 64
    sp, theta, src, dst = _register_setup(N, H, W, 3, precision)
    p = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)
    ll_fn = GaussianLogLikelihood(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.05,
                                  params_flow_int=p)
    ll = ll_fn.batch(torch.as_tensor(theta, device=DEV)).cpu().numpy()
    sA, Tr = sp.tables_from_theta(torch.as_tensor(theta, device=DEV), 0.02, -1)
    t = O.tess_struct(2, 1, (4, 4), sp.incs)
    for n in range(N):
        ll_o, _ = O.register_ll(t, Tr[n].cpu().numpy(), sA[n].cpu().numpy(), src[n], dst[n], 0.05, 0.02, 50, 100)
        assert abs(ll[n] - ll_o) <= rtol * abs(ll_o), (n, ll[n], ll_o)


def test_register_ll_same_alone_and_batched():
    N, H, W = 4, 48, 40
    sp, theta, src, dst = _register_setup(N, H, W, 4)
    p = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)
    full = GaussianLogLikelihood(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.05, p)
    ll_all = full.batch(torch.as_tensor(theta, device=DEV)).cpu().numpy()
    for n in range(N):
        one = GaussianLogLikelihood(sp, torch.as_tensor(src[n], device=DEV), torch.as_tensor(dst[n], device=DEV),
                                    0.05, p)
        assert one(theta[n]) == ll_all[n]


def test_register_ll_equals_unfused_path():
    """Fused likelihood == calc_T_inv of the grid, then remap_ssd (same tables)."""
    N, H, W = 2, 50, 60
    sp, theta, src, dst = _register_setup(N, H, W, 5)
    p = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)
    srcg, dstg = torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV)
    warped = torch.empty((N, H, W), dtype=torch.float32, device=DEV)
    ll = GaussianLogLikelihood(sp, srcg, dstg, 0.05, p).batch(torch.as_tensor(theta, device=DEV), warped=warped)
    grid = torch.as_tensor(pixel_centers(H, W), device=DEV)
    maps = torch.empty((N, H * W, 2), dtype=torch.float64, device=DEV)
    for n in range(N):
        sp.update_pat(sp.B @ torch.as_tensor(theta[n], device=DEV))
        sp.calc_T_inv(pts=grid, out=maps[n], **p)
    w2 = torch.empty_like(warped)
    ll2 = remap_ssd(maps, srcg, dstg, 0.05, pixel_map=UNIT(H, W), warped=w2)
    torch.testing.assert_close(warped, w2, rtol=0, atol=0)
    torch.testing.assert_close(ll, ll2, rtol=1e-12, atol=0)
