"""Voxel Eikonal, sign total variation and points loss on the GPU (the drop-in
``grid_loss_bw`` functions), against the reference's own CUDA outputs (tests/golden/reg.npz,
made by tests/golden/make_golden.py) and the C oracle."""
from __future__ import annotations

import functools

import numpy as np
import pytest
import torch

from svraster_b200 import grid_loss_bw as GL
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
