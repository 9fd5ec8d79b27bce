"""Pruning / subdivision kernels and the batched training statistics on the GPU, against the
reference's own torch code (golden vectors of tests/golden/make_golden_adaptive.py) and, for
the statistics, against per-view renders of the C oracle restating the reference's loop."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from svraster_b200 import adaptive as A
from svraster_b200 import synthetic as S
from tests.golden.adaptive_cases import OUTSIDE_LEVEL, model_inputs, scene

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "adaptive.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_grid_link_bitexact(gold):
    sc = scene()
    key, vkey = A.build_grid_pts_link(torch.from_numpy(sc.octpath).cuda(),
                                      torch.from_numpy(sc.octlevel.astype(np.int8)).cuda())
    assert np.array_equal(key.cpu().numpy(), gold["link_key"])
    assert np.array_equal(vkey.cpu().numpy(), gold["link_vox_key"])


def test_children_and_decoding(gold):
    sc = scene()
    sel = np.arange(0, sc.n_vox, 3)
    cp, cl = A.gen_children(torch.from_numpy(sc.octpath.reshape(-1, 1)[sel]).cuda(),
                            torch.from_numpy(sc.octlevel.reshape(-1, 1)[sel].astype(np.int8)).cuda())
    assert np.array_equal(cp.cpu().numpy(), gold["child_path"])
    assert np.array_equal(cl.cpu().numpy(), gold["child_level"])
    cc, cs = A.octpath_decoding(cp, cl, torch.zeros(3, device="cuda"), torch.tensor([2.0], device="cuda"))
    assert np.array_equal(cs.cpu().numpy(), gold["child_size"])
    np.testing.assert_allclose(cc.cpu().numpy(), gold["child_center"], rtol=0, atol=1e-7)


@pytest.mark.parametrize("c", [1, 3])
def test_subdivide_by_interp(gold, c):
    out = A.subdivide_by_interp(torch.from_numpy(gold[f"interp_in_{c}"]).cuda()).cpu().numpy()
    ref = gold[f"interp_out_{c}"]
    assert out.shape == ref.shape
    # every entry but the cube-centre mean is the reference's expression in its order
    np.testing.assert_allclose(out, ref, rtol=1e-6, atol=1e-7)
    child = np.arange(out.shape[0]) % 8
    for m in range(8):
        rows = child == m
        exact = [j for j in range(8) if j != m ^ 7]
        assert np.array_equal(out[rows][:, exact], ref[rows][:, exact])


def test_agg_voxel_into_grid_pts(gold):
    out = A.agg_voxel_into_grid_pts(len(gold["link_key"]), torch.from_numpy(gold["link_vox_key"]).cuda(),
                                    torch.from_numpy(gold["agg_in"]).cuda()).cpu().numpy()
    np.testing.assert_allclose(out, gold["agg_out"], rtol=1e-5, atol=1e-6)


class _Model(A.SVAdaptive):
    pass


def test_subdividing_then_pruning_matches_reference(gold):
    sc = scene()
    m = _Model()
    for k, v in model_inputs(sc).items():
        setattr(m, k, torch.from_numpy(v).cuda())
    m.scene_center, m.scene_extent = torch.zeros(3, device="cuda"), torch.tensor([2.0], device="cuda")
    m.outside_level = OUTSIDE_LEVEL
    m.per_voxel_attr_lst = ["octpath", "octlevel", "vox_center", "vox_size", "subdiv_meta", "is_leaf"]
    m.per_voxel_param_lst = ["_sh0", "_shs", "_subdiv_p"]
    m.grid_pts_param_lst = ["_geo_grid_pts"]
    m.grid_pts_key, m.vox_key = A.build_grid_pts_link(m.octpath, m.octlevel)
    m.subdividing(torch.from_numpy(np.random.default_rng(6).random(sc.n_vox) < 0.08).cuda())
    names = m.per_voxel_attr_lst + m.per_voxel_param_lst + ["vox_key", "grid_pts_key"]

    def check(prefix):
        for n in names:
            got, ref = getattr(m, n).detach().cpu().numpy(), gold[prefix + n]
            if n == "vox_center":
                np.testing.assert_allclose(got, ref, rtol=0, atol=1e-7, err_msg=prefix + n)
            else:
                assert np.array_equal(got, ref), prefix + n
        np.testing.assert_allclose(m._geo_grid_pts.detach().cpu().numpy(), gold[prefix + "_geo_grid_pts"],
                                   rtol=1e-5, atol=1e-6)
    check("sub_")
    m.pruning(torch.from_numpy(np.random.default_rng(7).random(len(m.octpath)) < 0.05).cuda())
    check("prune_")


def test_training_stat_matches_per_view_oracle():
    """Batched statistics vs the reference's per-camera loop over oracle renders."""
    from oracle import oracle as O
    sc = S.scene_small(seed=8)
    cams = S.ring_cameras(5, 3.0, 96, 72, fovx_deg=50.0, phase=0.4)
    dev = torch.device("cuda")
    geos = sc.geo_grid_pts.reshape(-1)[sc.vox_key]
    got = A.compute_training_stat(cams, torch.from_numpy(sc.octpath).to(dev), torch.from_numpy(sc.vox_center).to(dev),
                                  torch.from_numpy(sc.vox_size.reshape(-1, 1)).to(dev),
                                  torch.from_numpy(sc.is_leaf).to(dev), torch.from_numpy(geos).to(dev),
                                  torch.tensor([sc.s_val], device=dev))
    N = sc.n_vox
    max_w = np.zeros(N, np.float32)
    min_s = np.full(N, 1e30, np.float32)
    cnt = np.zeros(N, np.float32)
    for cam in cams:
        nd, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
        _, vals, ranges = O.binning(cam, sc.octpath, nd, bb, bits)
        f = O.render_fwd(cam, np.zeros(3, np.float32), 3, True, True, ranges, vals, bb, sc.vox_center, sc.vox_size,
                         geos, np.zeros((N, 3), np.float32), sc.s_val, track_max_w=True)
        mw = f["max_w"].reshape(-1)
        max_w = np.maximum(max_w, mw)
        vis = mw > 0
        look = cam.c2w[:3, 2].astype(np.float32)
        d = (sc.vox_center[vis] - cam.c2w[:3, 3].astype(np.float32)) * look
        z = (d[:, 0] + d[:, 1]) + d[:, 2]
        min_s[vis] = np.minimum(min_s[vis], z * np.float32(2 * cam.tanfovx / cam.width))
        cnt[vis] += 1
    g_mw = got["max_w"].cpu().numpy().reshape(-1)
    g_ms = got["min_samp_interval"].cpu().numpy().reshape(-1)
    g_cnt = got["view_cnt"].cpu().numpy().reshape(-1)
    np.testing.assert_allclose(g_mw, max_w, rtol=1e-4, atol=1e-6)
    # visibility decided by a weight > 0 can flip only for weights at the rounding level
    assert (g_cnt != cnt).mean() < 1e-3
    same = g_cnt == cnt
    np.testing.assert_allclose(g_ms[same], min_s[same], rtol=1e-6)
    assert cnt.max() >= 2
