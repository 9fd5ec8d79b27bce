"""Pin the oracle and the sm_100a library against golden vectors produced by the reference's
own CUDA extension (tests/golden/make_golden.py, run on a B200).

CPU tests check the C oracle against the goldens; GPU tests check the library.  Integer
stages (duplicate counts, bboxes, octant bits, sorted record order, tile ranges, dense-grid
table, Adam) must match bit for bit; floating-point outputs within the stated tolerances.
"""
import os

import numpy as np
import pytest

from tests.golden.cases import (ADAM_CASE, CASES, REG_CASE, TABLE_CASE, build_adam_inputs, build_case_inputs,
                                build_reg_inputs, build_table_inputs, digest)

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(HERE, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name}.npz not generated yet")
    return dict(np.load(path))


def _check_inputs(g, inp):
    assert str(g["digest"]) == digest(inp), "synthetic inputs changed; regenerate the golden fixtures"


def _flags(case, inp, geos, rgbs):
    """Pixels whose forward decisions sit at a threshold, from the oracle's trace of this case."""
    from oracle import oracle as O
    from tests.helpers import forward_flags
    sc, cam = inp["scene"], inp["cam"]
    nd, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
    _, vals, ranges = O.binning(cam, sc.octpath, nd, bb, bits)
    tr = np.zeros(cam.width * cam.height, np.uint8)
    O.set_trace(tr)
    try:
        O.render_fwd(cam, np.asarray(case["bg"], np.float32), case["vox_geo_mode"], True, True, ranges, vals, bb,
                     sc.vox_center, sc.vox_size, geos, rgbs, sc.s_val)
    finally:
        O.set_trace(None)
    return forward_flags(cam, tr)


def _compare_render(res, g, cam, flagged, tag):
    """Images against the reference's own extension on the pixels with no decision at a
    threshold (tests.helpers.image_parity: 1e-5 of the range everywhere, 1e-5 per element for
    99.8% of the entries); a decision at a threshold may move a pixel's last contributor."""
    from tests.helpers import images_match
    H, W = cam.height, cam.width
    got = {k: np.asarray(res[k]).reshape(ch, H, W) for k, ch in (("color", 3), ("T", 1), ("depth", 4), ("normal", 3))}
    images_match(got, g, flagged, tag)
    nc_bad = np.asarray(res["n_contrib"]).reshape(-1) != g["n_contrib"]
    assert not (nc_bad & ~flagged.reshape(-1)).any()


def _compare_grads(dvox, ds, g, n_vox):
    """Gradients: the same per-pair terms summed in another order (the reference adds with
    atomics in schedule order): within 1e-5 of the column's largest entry at the 99.9th
    percentile and 1e-4 everywhere; dL/ds (one sum over every pair) within 2e-5."""
    ref = np.zeros((n_vox, 12), np.float32)
    ref[g["dvox_rows"]] = g["dvox"]
    scale = np.abs(ref).max(0) + 1e-12
    err = np.abs(np.asarray(dvox) - ref) / scale
    assert np.quantile(err, 0.999) <= 1e-5, np.quantile(err, 0.999)
    assert err.max() <= 1e-4, err.max()
    assert abs(float(ds) - float(g["ds"][0])) <= 2e-5 * abs(float(g["ds"][0])) + 1e-7


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_reference_goldens(name):
    from oracle import oracle as O
    g = load(name)
    case = CASES[name]
    inp = build_case_inputs(case)
    _check_inputs(g, inp)
    sc, cam, grads = inp["scene"], inp["cam"], inp["grads"]
    nd, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
    assert np.array_equal(nd, g["n_dup"])
    # the reference leaves bbox / octant bits of culled voxels unwritten (torch::empty)
    r = nd > 0
    assert np.array_equal(bb[r], g["bbox"][r])
    assert np.array_equal(bits[r], g["bits"][r])
    keys, vals, ranges = O.binning(cam, sc.octpath, nd, bb, bits)
    assert int(g["num_rendered"]) == len(vals)
    assert np.array_equal(keys, g["keys"])
    assert np.array_equal(vals, g["vals"])
    ne = g["ranges"][:, 1] > g["ranges"][:, 0]
    assert np.array_equal(ranges[ne], g["ranges"][ne])
    care = g["care"]
    geos = O.gather_geo(care, sc.vox_key, sc.geo_grid_pts, sc.n_vox)
    assert np.array_equal(geos[care], g["geos"])
    rgbs = O.sh_eval(3, care, sc.vox_center, cam.position, sc.sh0, sc.shs)
    np.testing.assert_allclose(rgbs[care], g["rgbs"], rtol=2e-6, atol=2e-6)
    bg = np.asarray(case["bg"], np.float32)
    n_samp = {3: 3, 2: 2, 1: 1}[case["vox_geo_mode"]]
    f = O.render_fwd(cam, bg, n_samp, True, True, ranges, vals, bb, sc.vox_center, sc.vox_size, geos, rgbs,
                     sc.s_val, track_max_w=True)
    _compare_render(f, g, cam, _flags(case, inp, geos, rgbs), f"oracle {name}")
    dvox, ds = O.render_bwd(cam, bg, True, True, ranges, g["tile_last"], vals, bb, sc.vox_center, sc.vox_size, geos,
                            rgbs, sc.s_val, g["T"], g["n_contrib"], grads["color"], grads["depth"], grads["normal"],
                            grads["T"], case["lambda_R_concen"], grads["gt"])
    _compare_grads(dvox, ds, g, sc.n_vox)


def test_oracle_table_and_smoothness_match_reference_goldens():
    from oracle import oracle as O
    g = load("table")
    inp = build_table_inputs(TABLE_CASE)
    _check_inputs(g, inp)
    sc = inp["scene"]
    mask, keys, g2v = O.valid_table(sc.vox_center, sc.vox_size, np.zeros(3), sc.scene_extent,
                                    TABLE_CASE["res_pow2"], sc.is_leaf)
    assert np.array_equal(mask, g["mask"])
    assert np.array_equal(keys, g["keys"])
    assert np.array_equal(g2v, g["g2v"])
    res = 1 << TABLE_CASE["res_pow2"]
    for name, fn in (("lap", O.laplacian_bw), ("eik", O.eikonal_bw)):
        out = fn(sc.geo_grid_pts, sc.vox_key, inp["grid_voxel_coord"], inp["grid_voxel_size"], res, mask, keys, g2v,
                 inp["active"], TABLE_CASE["weight"], TABLE_CASE["vox_size_inv"], int(g["seed"]),
                 np.zeros((len(sc.geo_grid_pts), 1), np.float32)).reshape(-1)
        scale = np.abs(g[name]).max() + 1e-20
        assert np.abs(out - g[name]).max() <= 1e-4 * scale, name


def reg_outputs(inp, vg, tv, pl):
    """Run one implementation of the three regularisers on the regulariser case; ``vg``, ``tv``
    and ``pl`` take the reference argument order and return the updated gradient."""
    sc, tb, w = inp["scene"], inp["table"], REG_CASE["weight"]
    out = {"vg": vg(sc.geo_grid_pts, sc.vox_key, inp["vox_size_inv"], inp["active"], w, inp["grad1"])}
    for no_tv_s in (0, 1):
        for name, grid, g0 in (("1", sc.geo_grid_pts, inp["grad1"]), ("3", inp["grid3"], inp["grad3"])):
            out[f"tv{name}_{no_tv_s}"] = tv(grid, sc.vox_key, w, inp["vox_size_inv"], no_tv_s, False, g0)
    out["pl"] = pl(inp["points"], sc.geo_grid_pts, sc.vox_key, inp["grid_voxel_coord"], inp["grid_voxel_size"],
                   1 << REG_CASE["res_pow2"], tb["mask"], tb["keys"], tb["g2v"], w, inp["grad1"])
    return out


# The reference adds with float atomics in thread-schedule order; sums of the same terms in
# another order differ by a few ulps of the largest partial sum.
REG_RTOL, REG_ATOL = 1e-5, 1e-6


def check_reg(out, g):
    for k, v in out.items():
        ref = g[k]
        assert v.shape == ref.shape, k
        np.testing.assert_allclose(v, ref, rtol=REG_RTOL, atol=REG_ATOL * (np.abs(ref).max() + 1e-20), err_msg=k)


def test_oracle_regularisers_match_reference_goldens():
    from oracle import oracle as O
    g = load("reg")
    inp = build_reg_inputs(REG_CASE)
    _check_inputs(g, inp)
    out = reg_outputs(inp, O.voxel_gradient_bw, O.total_variation_bw, O.points_loss_bw)
    check_reg(out, g)
    # every output moved away from its starting gradient (the case exercises each path)
    assert (g["vg"] != inp["grad1"]).sum() > 1000 and (g["pl"] != inp["grad1"]).sum() > 1000
    assert (g["tv3_0"] != inp["grad3"]).mean() > 0.5


def test_oracle_sparse_total_variation_rule():
    """tv_sparse: a (voxel, channel) takes part iff one of its corners has a nonzero gradient on
    entry; planted on a two-voxel grid sharing a face."""
    from oracle import oracle as O
    # corners x<<2|y<<1|z of voxel 0 are grid points 0..7; voxel 1 is shifted by +x (points 4..11)
    key = np.array([[0, 1, 2, 3, 4, 5, 6, 7], [4, 5, 6, 7, 8, 9, 10, 11]], np.int64)
    grid = np.arange(12, dtype=np.float32).reshape(12, 1)
    vsi = np.ones(2, np.float32)
    zero = np.zeros((12, 1), np.float32)
    assert np.array_equal(O.total_variation_bw(grid, key, 1.0, vsi, 1, 1, zero), zero)
    g0 = zero.copy(); g0[9] = 0.5          # only voxel 1 has a nonzero corner
    dense = O.total_variation_bw(grid, key[1:], 1.0, vsi[1:], 1, 0, g0)
    assert np.array_equal(O.total_variation_bw(grid, key, 1.0, vsi, 1, 1, g0), dense)
    g0[4] = -1.0                           # a shared corner: both voxels take part
    assert np.array_equal(O.total_variation_bw(grid, key, 1.0, vsi, 1, 1, g0),
                          O.total_variation_bw(grid, key, 1.0, vsi, 1, 0, g0))


def test_oracle_adam_matches_reference_goldens():
    from oracle import oracle as O
    g = load("adam")
    inp = build_adam_inputs(ADAM_CASE)
    _check_inputs(g, inp)
    c = ADAM_CASE
    for biased in (False, True):
        for sparse in (False, True):
            k = f"{'b' if biased else 'u'}{'s' if sparse else 'd'}"
            p, m, v = O.adam(inp["param"], inp["grad"], inp["m"], inp["v"], c["step"], c["lr"], c["beta1"],
                             c["beta2"], c["eps"], biased=biased, sparse=sparse)
            np.testing.assert_array_equal(p, g[k + "_p"])
            np.testing.assert_array_equal(m, g[k + "_m"])
            np.testing.assert_array_equal(v, g[k + "_v"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_library_matches_reference_goldens(name):
    from tests.helpers import cuda_views
    g = load(name)
    case = CASES[name]
    inp = build_case_inputs(case)
    _check_inputs(g, inp)
    sc, cam, grads = inp["scene"], inp["cam"], inp["grads"]
    geos = np.zeros((sc.n_vox, 8), np.float32)
    geos[g["care"]] = g["geos"]
    rgbs = np.zeros((sc.n_vox, 3), np.float32)
    rgbs[g["care"]] = g["rgbs"]
    out = cuda_views(sc, [cam], geos, [rgbs], n_samp=case["vox_geo_mode"], bg=case["bg"], grads_list=[grads],
                     lambda_R=case["lambda_R_concen"])
    st = out["state"]
    nd, bb, bits = [x.cpu().numpy().view(np.uint32) for x in st.geom_fields()]
    assert np.array_equal(out["n_dup"].cpu().numpy(), g["n_dup"])
    r = g["n_dup"] > 0
    assert np.array_equal(bb.reshape(-1, 2)[r], g["bbox"][r])
    assert np.array_equal(bits[r], g["bits"][r])
    vals, ranges, tl, nc = [x.cpu().numpy().view(np.uint32) for x in st.binning_fields()]
    assert np.array_equal(vals, g["vals"]), "sorted record order differs from the reference"
    ne = g["ranges"][:, 1] > g["ranges"][:, 0]
    assert np.array_equal(ranges[ne], g["ranges"][ne])
    res = {k: out[k].cpu().numpy() for k in ("color", "T", "depth", "normal")}
    res["n_contrib"] = nc
    _compare_render(res, g, cam, _flags(case, inp, geos, rgbs), f"library {name}")
    _compare_grads(out["dvox"].cpu().numpy(), out["ds"].item(), g, sc.n_vox)
