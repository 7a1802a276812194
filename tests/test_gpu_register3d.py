"""3D remap (trilinear) and the fused 3D registration likelihood against the
oracle (C ABI underneath).

Tolerances: remapped volumes 1e-5 absolute; log-likelihoods 1e-12 relative
with float64 maps / FP64 integration (same points, same double arithmetic,
different summation order), 1e-6 relative with float32 maps / FP32
integration."""
import numpy as np
import pytest
import torch
from scipy.ndimage import gaussian_filter

from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.registration import GaussianLogLikelihood3D, TransformWrapper3D, remap3d, remap3d_ssd
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
P = dict(dt=0.02, nTimeSteps=50, nStepsODEsolver=100)


def unit(H, W, D):
    return (W, -0.5, H, -0.5, D, -0.5)


def smooth_volume(rng, H, W, D, sigma=2.0):
    return gaussian_filter(rng.uniform(0, 1, (H, W, D)).astype(np.float32), sigma, mode="reflect").astype(np.float32)


def voxel_centers(H, W, D):
    r, c, k = np.meshgrid(np.arange(H), np.arange(W), np.arange(D), indexing="ij")
    return np.stack([(c.ravel() + 0.5) / W, (r.ravel() + 0.5) / H, (k.ravel() + 0.5) / D], 1)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_remap3d_matches_oracle(oracle_mod, dt):
    O = oracle_mod
    rng = np.random.default_rng(0)
    H, W, D = 12, 17, 9
    vol = smooth_volume(rng, H, W, D)
    pts = voxel_centers(H, W, D) + rng.normal(0, 0.04, size=(H * W * D, 3))
    pts[:40] = rng.uniform(-0.3, 1.3, size=(40, 3))           # outside the volume too
    pts[40] = [np.nan, 0.5, 0.5]
    m = torch.as_tensor(pts, dtype=dt, device=DEV)
    got = remap3d(m, torch.as_tensor(vol, device=DEV), voxel_map=unit(H, W, D)).cpu().numpy()
    want = O.remap3d(m.cpu().numpy().astype(np.float64), vol, *unit(H, W, D))
    assert np.abs(got - want).max() < 1e-5


def test_remap3d_identity_voxel_units():
    rng = np.random.default_rng(1)
    H, W, D = 6, 5, 7
    vol = torch.as_tensor(rng.uniform(0, 1, (H, W, D)).astype(np.float32), device=DEV)
    r, c, k = np.meshgrid(np.arange(H), np.arange(W), np.arange(D), indexing="ij")
    m = torch.as_tensor(np.stack([c.ravel(), r.ravel(), k.ravel()], 1).astype(np.float64), device=DEV)
    assert torch.equal(remap3d(m, vol), vol)


@pytest.mark.parametrize("dt,rtol", [(torch.float64, 1e-12), (torch.float32, 1e-6)])
def test_remap3d_ssd_matches_oracle(oracle_mod, dt, rtol):
    O = oracle_mod
    rng = np.random.default_rng(2)
    N, H, W, D = 3, 10, 12, 14
    src = np.stack([smooth_volume(rng, H, W, D) for _ in range(N)])
    dst = np.stack([smooth_volume(rng, H, W, D) for _ in range(N)])
    pts = voxel_centers(H, W, D)[None] + rng.normal(0, 0.03, size=(N, H * W * D, 3))
    m = torch.as_tensor(pts, dtype=dt, device=DEV)
    warped = torch.empty((N, H, W, D), dtype=torch.float32, device=DEV)
    ll = remap3d_ssd(m, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.1,
                     voxel_map=unit(H, W, D), warped=warped).cpu().numpy()
    for n in range(N):
        ll_o, w_o = O.remap3d_ssd(m[n].cpu().numpy().astype(np.float64), src[n], dst[n], 0.1, *unit(H, W, D))
        assert abs(ll[n] - ll_o) <= rtol * abs(ll_o)
        assert np.abs(warped[n].cpu().numpy() - w_o).max() < 1e-5


def _register_setup(N, H, W, D, seed, precision=torch.float64):
    sp = CpaSpace([0.0] * 3, [1.0] * 3, (2, 2, 2), tess="I", device=DEV, precision=precision)
    rng = np.random.default_rng(seed)
    theta = Prior.create(sp.geo, 0.2, 0.5).sample(N, rng)
    src = np.stack([smooth_volume(rng, H, W, D) for _ in range(N)])
    dst = np.stack([smooth_volume(rng, H, W, D) for _ in range(N)])
    return sp, theta, src, dst


def _oracle_register3d(O, sp, tables, src, dst, H, W, D, sigma):
    sA, Tr = (x.cpu().numpy() for x in tables)
    t = O.tess_struct(3, sp.geo.tess_code, sp.geo.nCs, sp.geo.incs)
    grid = voxel_centers(H, W, D)
    out = []
    for n in range(sA.shape[0]):
        mp, _ = O.calc_T(t, Tr[n], sA[n], grid, P["dt"], P["nTimeSteps"], P["nStepsODEsolver"])
        out.append(O.remap3d_ssd(mp, src[n], dst[n], sigma, *unit(H, W, D))[0])
    return np.array(out)


@pytest.mark.parametrize("precision,rtol", [(torch.float64, 1e-12), (torch.float32, 1e-6)])
def test_register3d_ll_matches_oracle(oracle_mod, precision, rtol):
    N, H, W, D = 2, 10, 11, 12
    sp, theta, src, dst = _register_setup(N, H, W, D, 3, precision)
    f = GaussianLogLikelihood3D(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV), 0.05, P)
    tables = sp.tables_from_theta(torch.as_tensor(theta, device=DEV), P["dt"], -1)
    ll = f.batch_tables(tables).cpu().numpy()
    ll_o = _oracle_register3d(oracle_mod, sp, tables, src, dst, H, W, D, 0.05)
    np.testing.assert_allclose(ll, ll_o, rtol=rtol)


def test_register3d_equals_unfused_path():
    """Fused likelihood == calc_T_inv of the voxel grid, then remap3d_ssd (same tables)."""
    N, H, W, D = 2, 8, 9, 10
    sp, theta, src, dst = _register_setup(N, H, W, D, 4)
    srcg, dstg = torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV)
    warped = torch.empty((N, H, W, D), dtype=torch.float32, device=DEV)
    ll = GaussianLogLikelihood3D(sp, srcg, dstg, 0.05, P).batch(torch.as_tensor(theta, device=DEV), warped=warped)
    grid = torch.as_tensor(voxel_centers(H, W, D), device=DEV)
    maps = torch.empty((N, H * W * D, 3), dtype=torch.float64, device=DEV)
    for n in range(N):
        sp.update_pat(sp.B @ torch.as_tensor(theta[n], device=DEV))
        sp.calc_T_inv(pts=grid, out=maps[n], **P)
    w2 = torch.empty_like(warped)
    ll2 = remap3d_ssd(maps, srcg, dstg, 0.05, voxel_map=unit(H, W, D), warped=w2)
    torch.testing.assert_close(warped, w2, rtol=0, atol=0)
    torch.testing.assert_close(ll, ll2, rtol=1e-12, atol=0)


def test_register3d_same_alone_and_batched():
    N, H, W, D = 3, 9, 8, 30                     # several tiles per volume
    sp, theta, src, dst = _register_setup(N, H, W, D, 5)
    th = torch.as_tensor(theta, device=DEV)
    batched = GaussianLogLikelihood3D(sp, torch.as_tensor(src, device=DEV), torch.as_tensor(dst, device=DEV),
                                      0.05, P).batch(th)
    for n in range(N):
        alone = GaussianLogLikelihood3D(sp, torch.as_tensor(src[n], device=DEV), torch.as_tensor(dst[n], device=DEV),
                                        0.05, P).batch(th[n:n + 1])
        assert torch.equal(alone[0], batched[n])


def test_transform_wrapper3d_identity_remap():
    tw = TransformWrapper3D(6, 7, 5, base=(2, 2, 2), tess="II", device=DEV)
    rng = np.random.default_rng(6)
    vol = torch.as_tensor(rng.uniform(0, 1, (6, 7, 5)).astype(np.float32), device=DEV)
    tw.update_pat_from_theta(np.zeros(tw.space.d))
    pts_inv = torch.empty_like(tw.pts_src_dense)
    tw.calc_T_inv(tw.pts_src_dense, pts_inv)
    out = torch.empty_like(vol)
    tw.remap_fwd(pts_inv, vol, out)
    assert torch.equal(pts_inv, tw.pts_src_dense)
    assert torch.equal(out, vol)
