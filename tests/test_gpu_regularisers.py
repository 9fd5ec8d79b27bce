"""Voxel Eikonal, sign total variation and points loss on the GPU (the drop-in
``grid_loss_bw`` functions), against the reference's own CUDA outputs (tests/golden/reg.npz,
made by tests/golden/make_golden.py) and the C oracle."""
from __future__ import annotations

import functools

import numpy as np
import pytest
import torch

from svraster_b200 import grid_loss_bw as GL
from svraster_b200 import synthetic as S
from tests.golden.cases import REG_CASE, build_reg_inputs
from tests.test_golden import _check_inputs, check_reg, load, reg_outputs

pytestmark = pytest.mark.gpu


def cu(a, dt=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t if dt is None else t.to(dt)


def gpu_vg(grid, key, vsi, active, w, g0, ordered=True):
    g = cu(g0)
    GL.voxel_gradient(cu(grid), cu(key), cu(vsi), cu(active), w, False, False, g, check_status=True, ordered=ordered)
    return g.cpu().numpy()


def gpu_tv(grid, key, w, vsi, no_tv_s, tv_sparse, g0, ordered=True):
    g = cu(g0)
    GL.total_variation(cu(grid), cu(key), w, cu(vsi), bool(no_tv_s), bool(tv_sparse), g, check_status=True,
                       ordered=ordered)
    return g.cpu().numpy()


def gpu_pl(points, grid, key, coord, size, res, mask, keys, g2v, w, g0, use_index=True):
    g = cu(g0)
    GL.points_loss(cu(points), cu(grid), cu(key), cu(coord), cu(size), res, cu(mask, torch.bool), cu(keys),
                   cu(g2v), w, 1.0, True, False, g, use_index=use_index, check_status=True)
    return g.cpu().numpy()


@pytest.fixture(scope="module")
def case():
    return build_reg_inputs(REG_CASE)


@pytest.mark.parametrize("ordered", [True, False], ids=["spatial-order", "storage-order"])
def test_library_matches_reference_goldens(case, ordered):
    """The case's voxel list has repeats (a voxel listed twice adds twice in both forms)."""
    g = load("reg")
    _check_inputs(g, case)
    check_reg(reg_outputs(case, functools.partial(gpu_vg, ordered=ordered),
                          functools.partial(gpu_tv, ordered=ordered), gpu_pl), g)


def test_voxel_order_is_stable_sort_of_first_corner():
    """order = stable argsort of vox_key[:, 0], rank its inverse (bit-exact)."""
    sc = build_reg_inputs(REG_CASE)["scene"]
    order, rank = GL.voxel_order(cu(sc.vox_key), sc.geo_grid_pts.shape[0])
    ref = np.argsort(sc.vox_key[:, 0], kind="stable").astype(np.int32)
    assert np.array_equal(order.cpu().numpy(), ref)
    inv = np.empty_like(ref)
    inv[ref] = np.arange(len(ref), dtype=np.int32)
    assert np.array_equal(rank.cpu().numpy(), inv)


@pytest.mark.parametrize("ordered", [True, False], ids=["spatial-order", "storage-order"])
@pytest.mark.parametrize("no_tv_s", [0, 1])
@pytest.mark.parametrize("ch", ["1", "3"])
def test_sparse_total_variation_matches_oracle(case, no_tv_s, ch, ordered):
    """tv_sparse decides participation from the gradient on entry, as the oracle does."""
    from oracle import oracle as O
    sc = case["scene"]
    grid, g0 = (sc.geo_grid_pts, case["grad1"]) if ch == "1" else (case["grid3"], case["grad3"])
    args = (grid, sc.vox_key, REG_CASE["weight"], case["vox_size_inv"], no_tv_s, 1, g0)
    got, ref = gpu_tv(*args, ordered=ordered), O.total_variation_bw(*args)
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
    dense = O.total_variation_bw(grid, sc.vox_key, REG_CASE["weight"], case["vox_size_inv"], no_tv_s, 0, g0)
    assert not np.array_equal(ref, dense)     # the sparse rule skipped some voxels


def test_empty_inputs_leave_gradient_alone(case):
    sc = case["scene"]
    g0 = case["grad1"]
    assert np.array_equal(gpu_vg(sc.geo_grid_pts, sc.vox_key, case["vox_size_inv"], np.zeros(0, np.int32), 0.01, g0),
                          g0)
    assert np.array_equal(gpu_tv(sc.geo_grid_pts, sc.vox_key[:0], 0.01, case["vox_size_inv"][:0], 0, 0, g0), g0)
    tb = case["table"]
    assert np.array_equal(gpu_pl(np.zeros((0, 3), np.float32), sc.geo_grid_pts, sc.vox_key,
                                 case["grid_voxel_coord"], case["grid_voxel_size"], 32, tb["mask"], tb["keys"],
                                 tb["g2v"], 0.01, g0), g0)


@pytest.mark.parametrize("ordered", [True, False], ids=["spatial-order", "storage-order"])
def test_out_of_range_voxel_is_reported(case, ordered):
    sc = case["scene"]
    bad = np.array([0, sc.n_vox + 5], np.int32)
    with pytest.raises(RuntimeError, match="status"):
        gpu_vg(sc.geo_grid_pts, sc.vox_key, case["vox_size_inv"], bad, 0.01, case["grad1"], ordered=ordered)


@pytest.mark.parametrize("ordered", [True, False], ids=["spatial-order", "storage-order"])
def test_larger_scene_matches_oracle(ordered):
    """53k voxels / 75k grid points: voxel Eikonal on a random half of the voxels, total
    variation on 1 and 4 channels (both no_tv_s), against the oracle."""
    from oracle import oracle as O
    sc = S.scene_small(seed=4)
    rng = np.random.default_rng(12)
    N, M = sc.n_vox, sc.geo_grid_pts.shape[0]
    vsi = (1.0 / sc.vox_size.reshape(-1)).astype(np.float32)
    active = rng.permutation(N)[:N // 2].astype(np.int32)
    g0 = np.where(rng.random((M, 1)) < 0.05, rng.normal(size=(M, 1)), 0).astype(np.float32)
    ref = O.voxel_gradient_bw(sc.geo_grid_pts, sc.vox_key, vsi, active, 1e-3, g0)
    got = gpu_vg(sc.geo_grid_pts, sc.vox_key, vsi, active, 1e-3, g0, ordered=ordered)
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
    grid4 = rng.normal(size=(M, 4)).astype(np.float32)
    g4 = np.zeros((M, 4), np.float32)
    for grid, g in ((sc.geo_grid_pts, g0), (grid4, g4)):
        for no_tv_s in (0, 1):
            ref = O.total_variation_bw(grid, sc.vox_key, 1e-3, vsi, no_tv_s, 0, g)
            got = gpu_tv(grid, sc.vox_key, 1e-3, vsi, no_tv_s, 0, g, ordered=ordered)
            np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())


def test_points_loss_larger_scene_matches_oracle():
    """200k points on the 53k-voxel scene's dense table, both key lookups, against the oracle."""
    from oracle import oracle as O
    from tests.golden.cases import grid_voxel_geometry
    sc = S.scene_small(seed=4)
    res_pow2 = int(sc.octlevel.max())
    res = 1 << res_pow2
    coord, size = grid_voxel_geometry(sc, res_pow2)
    mask, keys, g2v = O.valid_table(sc.vox_center, sc.vox_size, np.zeros(3, np.float32), sc.scene_extent, res_pow2,
                                    sc.is_leaf)
    rng = np.random.default_rng(13)
    cells = np.flatnonzero(mask)
    pick = cells[rng.integers(0, len(cells), size=200000)]
    pts = (np.stack([pick % res, (pick // res) % res, pick // (res * res)], 1) + rng.random((200000, 3)))
    pts = pts.astype(np.float32)
    g0 = np.zeros_like(sc.geo_grid_pts)
    ref = O.points_loss_bw(pts, sc.geo_grid_pts, sc.vox_key, coord, size, res, mask, keys, g2v, 1e-3, g0)
    for use_index in (True, False):
        got = gpu_pl(pts, sc.geo_grid_pts, sc.vox_key, coord, size, res, mask, keys, g2v, 1e-3, g0,
                     use_index=use_index)
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
