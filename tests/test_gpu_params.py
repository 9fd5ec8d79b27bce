"""Gather / SH / Adam / dense-grid table / smoothness adjoints: sm_100a library (through the
C ABI) against the C oracle on the same seeded inputs."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from svraster_b200 import _lib, grid_loss_bw, utils
from svraster_b200 import synthetic as S
from svraster_b200._lib import check, ptr, stream_ptr
from tests.golden.cases import grid_voxel_geometry

pytestmark = pytest.mark.gpu
dev = torch.device("cuda")


def T(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)


def test_gather_and_adjoint_bitexact():
    sc = S.scene_small(seed=1)
    rng = np.random.default_rng(0)
    care = np.sort(rng.choice(sc.n_vox, sc.n_vox // 3, replace=False)).astype(np.int64)
    geos = torch.zeros(sc.n_vox, 8, device=dev)
    L = _lib.load()
    # every tensor handed to the C ABI must outlive the call: bind them to names
    care_t, key_t, grid_t = T(care, torch.int64), T(sc.vox_key, torch.int64), T(sc.geo_grid_pts)
    check(L.svr_gather_geo(len(care), ptr(care_t), ptr(key_t), ptr(grid_t), ptr(geos), stream_ptr()), "gather")
    ref = O.gather_geo(care, sc.vox_key, sc.geo_grid_pts, sc.n_vox)
    assert np.array_equal(geos.cpu().numpy()[care], ref[care])
    dgeos = rng.normal(size=(sc.n_vox, 8)).astype(np.float32)
    dgrid = torch.zeros(len(sc.geo_grid_pts), 1, device=dev)
    dgeos_t = T(dgeos)
    check(L.svr_gather_geo_bw(len(care), ptr(care_t), ptr(key_t), ptr(dgeos_t), ptr(dgrid), stream_ptr()),
          "gather_bw")
    refg = O.gather_geo_bw(care, sc.vox_key, dgeos, len(sc.geo_grid_pts))
    np.testing.assert_allclose(dgrid.cpu().numpy(), refg, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_sh_eval_and_adjoint(deg):
    sc = S.scene_small(seed=2)
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(sc.n_vox, 5000, replace=False)).astype(np.int64)
    cam_pos = np.array([2.5, -1.0, 1.2], np.float32)
    from svraster_b200.renderer import SH_eval
    sh0 = T(sc.sh0).requires_grad_(True)
    shs = T(sc.shs).requires_grad_(True)
    rgbs = SH_eval.apply(deg, T(idx, torch.int64), T(sc.vox_center), T(cam_pos), None, sh0, shs)
    ref = O.sh_eval(deg, idx, sc.vox_center, cam_pos, sc.sh0, sc.shs)
    np.testing.assert_allclose(rgbs.detach().cpu().numpy(), ref, rtol=2e-6, atol=2e-6)
    d = rng.normal(size=(sc.n_vox, 3)).astype(np.float32)
    rgbs.backward(T(d))
    r0, r1 = O.sh_eval_bw(deg, idx, sc.vox_center, cam_pos, d, 16)
    np.testing.assert_allclose(sh0.grad.cpu().numpy(), r0, rtol=2e-6, atol=2e-6)
    np.testing.assert_allclose(shs.grad.cpu().numpy(), r1, rtol=2e-6, atol=2e-6)


@pytest.mark.parametrize("biased,sparse", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("n", [1, 7, 4099])
def test_adam_bitexact(biased, sparse, n):
    rng = np.random.default_rng(n)
    p, g = rng.normal(size=n).astype(np.float32), rng.normal(size=n).astype(np.float32)
    g[rng.random(n) < 0.3] = 0
    m, v = (0.1 * rng.normal(size=n)).astype(np.float32), np.abs(rng.normal(size=n)).astype(np.float32)
    pt, mt, vt, gt = T(p), T(m), T(v), T(g)
    check(_lib.load().svr_adam_step(n, int(biased), int(sparse), ptr(pt), ptr(gt), ptr(mt), ptr(vt), 5.0, 0.01, 0.1,
                                    0.99, 1e-15, stream_ptr()), "adam")
    rp, rm, rv = O.adam(p, g, m, v, 5, 0.01, 0.1, 0.99, 1e-15, biased=biased, sparse=sparse)
    np.testing.assert_array_equal(pt.cpu().numpy(), rp)
    np.testing.assert_array_equal(mt.cpu().numpy(), rm)
    np.testing.assert_array_equal(vt.cpu().numpy(), rv)


def _table(sc, res_pow2):
    mask, keys, g2v = utils.valid_gradient_table(T(sc.vox_center), T(sc.vox_size), T(np.zeros(3)), sc.scene_extent,
                                                 res_pow2, T(sc.is_leaf, torch.uint8))
    return mask, keys, g2v


@pytest.mark.parametrize("kind,res_pow2", [("tiny", 5), ("small", 7), ("small", 6)])
def test_valid_table_bitexact(kind, res_pow2):
    sc = S.scene_tiny() if kind == "tiny" else S.scene_small()
    mask, keys, g2v = _table(sc, res_pow2)
    rm, rk, rv = O.valid_table(sc.vox_center, sc.vox_size, np.zeros(3), sc.scene_extent, res_pow2, sc.is_leaf)
    assert np.array_equal(mask.cpu().numpy(), rm)
    assert np.array_equal(keys.cpu().numpy(), rk)
    assert np.array_equal(g2v.cpu().numpy(), rv)


@pytest.mark.parametrize("use_index", [True, False])
@pytest.mark.parametrize("which", ["lap", "eik"])
def test_smoothness_adjoints_match_oracle(which, use_index):
    sc = S.scene_small(seed=3)
    res_pow2 = 7
    mask, keys, g2v = _table(sc, res_pow2)
    coord, vsize = grid_voxel_geometry(sc, res_pow2)
    rng = np.random.default_rng(4)
    G = keys.numel()
    active = rng.permutation(G)[: G // 2].astype(np.int32)
    grad = torch.zeros(len(sc.geo_grid_pts), 1, device=dev)
    fn = grid_loss_bw.laplacian_smoothness if which == "lap" else grid_loss_bw.grid_eikonal
    fn(T(sc.geo_grid_pts), T(sc.vox_key, torch.int64), T(coord), T(vsize), 1 << res_pow2, mask, keys, g2v,
       T(active, torch.int32), 0.01, float(1 << res_pow2) / sc.scene_extent, True, False, grad, seed=777,
       use_index=use_index)
    ofn = O.laplacian_bw if which == "lap" else O.eikonal_bw
    ref = ofn(sc.geo_grid_pts, sc.vox_key, coord, vsize, 1 << res_pow2, mask.cpu().numpy(), keys.cpu().numpy(),
              g2v.cpu().numpy(), active, 0.01, float(1 << res_pow2) / sc.scene_extent, 777,
              np.zeros((len(sc.geo_grid_pts), 1), np.float32))
    g = grad.cpu().numpy()
    scale = np.abs(ref).max() + 1e-20
    assert np.abs(g - ref).max() <= 1e-4 * scale + 1e-7
    assert np.abs(ref).sum() > 0
