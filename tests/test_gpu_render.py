"""Parity of the sm_100a rasterizer (through the C ABI) with the C oracle on the same
seeded inputs: integer stages bit-exact, floating-point outputs within tolerance."""
import numpy as np
import pytest
import torch

from tests.helpers import (assert_close, cuda_views, images_match, oracle_inputs, oracle_view, scene_and_cams,
                           split_view, upstream_grads)

pytestmark = pytest.mark.gpu

# Images: tests.helpers.image_parity on the pixels with no decision at a threshold (1e-5 of the
# channel's range everywhere, 1e-5 per element for all but 0.2% of the entries above 1% of the
# range); such a decision may move a pixel's last contributor, nothing else may.


@pytest.mark.parametrize("kind,W,H,n_cams", [("tiny", 64, 48, 2), ("tiny", 130, 70, 1), ("small", 256, 256, 2)])
def test_preprocess_and_binning_bitexact(kind, W, H, n_cams):
    sc, cams = scene_and_cams(kind, n_cams, W, H)
    for cam in cams:
        geos, rgbs = oracle_inputs(sc, cam)
        ref = oracle_view(sc, cam, geos, rgbs)
        out = cuda_views(sc, [cam], geos, [rgbs])
        st = out["state"]
        nd, bb, bits = [x.cpu().numpy() for x in st.geom_fields()]
        assert np.array_equal(out["n_dup"].cpu().numpy(), ref["n_dup"])
        assert np.array_equal(nd.astype(np.uint32), ref["n_dup"].astype(np.uint32))
        assert np.array_equal(bb.view(np.uint32), ref["bbox"])
        assert np.array_equal(bits.view(np.uint32), ref["bits"])
        vals, ranges, tl, nc = [x.cpu().numpy().view(np.uint32) for x in st.binning_fields()]
        assert st.num_rendered == len(ref["vals"])
        assert np.array_equal(vals, ref["vals"]), "sorted record order differs"
        nonempty = ref["ranges"][:, 1] > ref["ranges"][:, 0]
        assert np.array_equal(ranges[nonempty], ref["ranges"][nonempty])
        assert st.status() == 0


@pytest.mark.parametrize("n_samp", [3, 2, 1])
def test_render_forward_matches_oracle(n_samp):
    sc, cams = scene_and_cams("small", 1, 200, 150)
    cam = cams[0]
    geos, rgbs = oracle_inputs(sc, cam)
    ref = oracle_view(sc, cam, geos, rgbs, n_samp=n_samp, bg=(0.2, 0.3, 0.4))
    out = cuda_views(sc, [cam], geos, [rgbs], n_samp=n_samp, bg=(0.2, 0.3, 0.4), track_max_w=True)
    H, W = cam.height, cam.width
    got = {k: out[k].cpu().numpy().reshape(ch, H, W) for k, ch in (("color", 3), ("T", 1), ("depth", 4), ("normal", 3))}
    images_match(got, ref, ref["flags"], f"n_samp {n_samp}")
    assert_close("max_w", out["max_w"].cpu().numpy(), ref["max_w"].reshape(-1), 1e-5, 1e-7, 1e-3)
    _, _, tl, nc = [x.cpu().numpy().view(np.uint32) for x in out["state"].binning_fields()]
    assert not ((nc != ref["n_contrib"]) & ~ref["flags"].reshape(-1)).any()
    assert (tl != ref["tile_last"]).mean() <= 0.05


@pytest.mark.parametrize("lambda_R", [0.0, 0.1])
def test_render_backward_matches_oracle(lambda_R):
    sc, cams = scene_and_cams("small", 1, 160, 120, seed=2)
    cam = cams[0]
    geos, rgbs = oracle_inputs(sc, cam)
    grads = upstream_grads(cam.height, cam.width, seed=5)[0]
    ref = oracle_view(sc, cam, geos, rgbs, grads=grads, lambda_R=lambda_R)
    out = cuda_views(sc, [cam], geos, [rgbs], grads_list=[grads], lambda_R=lambda_R)
    dv = out["dvox"].cpu().numpy()
    scale = np.abs(ref["dvox"]).max(0) + 1e-12
    # per-column relative-to-max comparison: the sums run in a different order (atomics), and
    # the device's expf and the host's differ by an ulp
    err = np.abs(dv - ref["dvox"]) / scale
    assert np.quantile(err, 0.999) <= 1e-5, np.quantile(err, 0.999)
    assert err.max() <= 1e-3, err.max()
    assert abs(out["ds"].item() - ref["ds"]) <= 1e-4 * abs(ref["ds"]) + 1e-6


def test_batched_views_equal_per_view():
    sc, cams = scene_and_cams("small", 3, 96, 80, seed=3)
    cams[1] = scene_and_cams("small", 1, 150, 60, seed=4)[1][0]
    gr = upstream_grads(1, 1)  # unused shape placeholder
    geos, _ = oracle_inputs(sc, cams[0])
    rgbs = [oracle_inputs(sc, c)[1] for c in cams]
    grads = [upstream_grads(c.height, c.width, seed=10 + i)[0] for i, c in enumerate(cams)]
    batch = cuda_views(sc, cams, geos, rgbs, grads_list=grads)
    dvox_sum = np.zeros((sc.n_vox, 12), np.float64)
    drgb_batch = batch["drgbs"].cpu().numpy().reshape(len(cams), sc.n_vox, 3)
    for v, cam in enumerate(cams):
        single = cuda_views(sc, [cam], geos, [rgbs[v]], grads_list=[grads[v]])
        for key, ch in (("color", 3), ("depth", 4), ("normal", 3), ("T", 1)):
            a = split_view(batch[key].cpu().numpy(), cams, v, ch)
            b = single[key].cpu().numpy().reshape(ch, cam.height, cam.width)
            assert np.array_equal(a, b), f"view {v} {key} differs between batched and per-view launch"
        d1 = single["dvox"].cpu().numpy()
        dvox_sum += d1
        np.testing.assert_allclose(drgb_batch[v], d1[:, 8:11], rtol=1e-4, atol=1e-4)
    db = batch["dvox"].cpu().numpy()
    np.testing.assert_allclose(db[:, :8], dvox_sum[:, :8], rtol=1e-3, atol=1e-2)


def test_mixed_resolution_batch_matches_oracle():
    """One launch over views of the batched configuration's four aspect ratios (scaled down,
    shuffled, none a multiple of the 16-pixel tile): every view equals the oracle's render of
    that view alone, in the heavy-tile-first launch order."""
    from svraster_b200 import synthetic as S
    sc = S.scene_small(seed=6)
    sizes = [(60, 45), (120, 68), (160, 90), (240, 135)]
    pos = S.fibonacci_points(4, 3.0)
    cams = [S.look_at_camera(pos[i], *sizes[k]) for i, k in enumerate((2, 0, 3, 1))]
    geos, _ = oracle_inputs(sc, cams[0])
    rgbs = [oracle_inputs(sc, c)[1] for c in cams]
    out = cuda_views(sc, cams, geos, rgbs)
    for v, cam in enumerate(cams):
        ref = oracle_view(sc, cam, geos, rgbs[v])
        got = {key: split_view(out[key].cpu().numpy(), cams, v, ch)
               for key, ch in (("color", 3), ("T", 1), ("depth", 4), ("normal", 3))}
        images_match(got, ref, ref["flags"], f"view {v}")


def test_empty_view_and_all_culled():
    sc, cams = scene_and_cams("tiny", 1, 64, 48)
    # camera looking away from the scene: nothing rendered, background everywhere
    from svraster_b200 import synthetic as S
    cam = S.look_at_camera([3.0, 0.0, 0.0], 64, 48, target=(6.0, 0.0, 0.0))
    geos, rgbs = oracle_inputs(sc, cam)
    out = cuda_views(sc, [cam], geos, [rgbs], bg=(0.5, 0.25, 0.125),
                     grads_list=upstream_grads(48, 64))
    assert out["state"].num_rendered == 0
    T = out["T"].cpu().numpy()
    assert np.all(T == 1.0)
    c = out["color"].cpu().numpy().reshape(3, -1)
    assert np.allclose(c[0], 0.5) and np.allclose(c[1], 0.25) and np.allclose(c[2], 0.125)
    assert float(out["dvox"].abs().sum()) == 0.0


def test_pair_counting_instance_matches_forward():
    """The counting instance of the forward writes the same images bit for bit, and its pair
    counts are ordered: accepted <= evaluated up to the last contributor <= evaluated."""
    sc, cams = scene_and_cams("small", 2, 160, 120, seed=7)
    geos, _ = oracle_inputs(sc, cams[0])
    rgbs = [oracle_inputs(sc, c)[1] for c in cams]
    out = cuda_views(sc, cams, geos, rgbs)
    st = out["state"]
    s_val = torch.tensor([sc.s_val], dtype=torch.float32, device="cuda")
    (n_eval, n_acc, n_last), planes = st.count_pairs(s_val, return_planes=True)
    assert 0 < n_acc <= n_last <= n_eval
    for a, k in zip(planes, ("color", "depth", "normal", "T")):
        assert torch.equal(a, out[k]), k
