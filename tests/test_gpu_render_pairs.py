"""The pair-evaluating render kernels (record-parallel filter, dense pair evaluation) against
the warp-filter kernels on the same binned records: the forward's outputs are bit-identical
(colour, depth, normal, transmittance, last contributors, tile ends, max weight) and the
adjoint's gradients agree up to the order of their float atomics."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from svraster_b200 import _lib
from svraster_b200 import synthetic as S
from tests.helpers import cam_dict, oracle_inputs, torch_scene, upstream_grads

pytestmark = pytest.mark.gpu


def _impl():
    f, b = C.c_int(0), C.c_int(0)
    _lib.load().svr_render_get_impl(C.byref(f), C.byref(b))
    return f.value, b.value


def _render_both(sc, cams, track_max_w=False, grads=None):
    from svraster_b200.raster import RasterState
    ts = torch_scene(sc)
    views = [cam_dict(c) for c in cams]
    st = RasterState(views, sc.n_vox, torch.device("cuda"))
    st.preprocess(ts["octpath"], ts["centers"], ts["lengths"], ts["is_leaf"])
    st.bin(ts["octpath"])
    geos = torch.as_tensor(oracle_inputs(sc, cams[0])[0]).cuda()
    rgbs = torch.as_tensor(np.concatenate([oracle_inputs(sc, c)[1] for c in cams], 0)).cuda()
    s_val = torch.tensor([sc.s_val], dtype=torch.float32, device="cuda")
    L = _lib.load()
    saved = _impl()
    outs = []
    try:
        for impl in (0, 1, 2, 3):
            assert L.svr_render_set_impl(impl, saved[1]) == 0
            o = st.render(3, True, True, ts["centers"], ts["lengths"], geos, rgbs, s_val, track_max_w=track_max_w,
                          rgb_per_view=len(cams) > 1)
            _, _, tl, nc = st.binning_fields()
            outs.append([x.clone() if x is not None else None for x in o] + [tl.clone(), nc.clone()])
            assert st.status() == 0
    finally:
        L.svr_render_set_impl(*saved)
    return outs


@pytest.mark.parametrize("kind,n_cams,W,H,seed", [("small", 2, 200, 150, 1), ("small", 1, 333, 257, 2),
                                                  ("small", 2, 40, 24, 3), ("tiny", 3, 64, 48, 0)])
def test_pair_forward_is_bit_identical(kind, n_cams, W, H, seed):
    sc = S.scene_small(seed=seed) if kind == "small" else S.scene_tiny(seed=seed)
    cams = S.ring_cameras(n_cams, 3.0, W, H, fovx_deg=50.0, phase=0.4 * seed)
    a, *others = _render_both(sc, cams, track_max_w=True)
    names = ("color", "depth", "normal", "T", "max_w", "tile_last", "n_contrib")
    for impl, b in enumerate(others, 1):
        for name, x, y in zip(names, a, b):
            assert torch.equal(x, y), f"{name} differs between the kernels (impl {impl})"


def test_pair_forward_bit_identical_mid_size_workload():
    import bench
    sc, cams = bench.make_workload(0, config="mid")
    a, *others = _render_both(sc, cams[:4])
    for impl, b in enumerate(others, 1):
        for name, x, y in zip(("color", "depth", "normal", "T", "max_w", "tile_last", "n_contrib"), a, b):
            if x is not None:
                assert torch.equal(x, y), f"{name} differs between the kernels (impl {impl})"


def _adjoint_both(sc, cams, lambda_R):
    from svraster_b200.raster import RasterState
    ts = torch_scene(sc)
    views = [cam_dict(c) for c in cams]
    st = RasterState(views, sc.n_vox, torch.device("cuda"))
    st.preprocess(ts["octpath"], ts["centers"], ts["lengths"], ts["is_leaf"])
    st.bin(ts["octpath"])
    geos = torch.as_tensor(oracle_inputs(sc, cams[0])[0]).cuda()
    rgbs = torch.as_tensor(np.concatenate([oracle_inputs(sc, c)[1] for c in cams], 0)).cuda()
    s_val = torch.tensor([sc.s_val], dtype=torch.float32, device="cuda")
    color, depth, normal, T, _ = st.render(3, True, True, ts["centers"], ts["lengths"], geos, rgbs, s_val,
                                           rgb_per_view=len(cams) > 1)
    gr = [upstream_grads(c.height, c.width, seed=20 + i)[0] for i, c in enumerate(cams)]
    cat = lambda k: torch.as_tensor(np.concatenate([g[k].reshape(-1) for g in gr])).cuda().float()
    L = _lib.load()
    saved = _impl()
    outs = []
    try:
        for impl in (0, 1, 2, 3):
            assert L.svr_render_set_impl(saved[0], impl) == 0
            drgbs = torch.zeros(len(cams) * sc.n_vox, 3, device="cuda") if len(cams) > 1 else None
            dvox, ds = st.render_backward(True, True, s_val, T, cat("color"), cat("depth"), cat("normal"), cat("T"),
                                          lambda_R_concen=lambda_R, gt_color=cat("gt") if lambda_R > 0 else None,
                                          drgbs=drgbs)
            torch.cuda.synchronize()
            assert st.status() == 0
            outs.append((dvox.cpu().numpy(), float(ds.item()), None if drgbs is None else drgbs.cpu().numpy()))
    finally:
        L.svr_render_set_impl(*saved)
    return outs


def _close_sums(a, b, name):
    """Equal up to the order of float additions: within 1e-5 of the column's largest entry."""
    scale = np.abs(b).max(0) + 1e-30
    err = np.abs(a - b) / scale
    assert err.max() < 1e-5, (name, float(err.max()))


@pytest.mark.parametrize("kind,n_cams,W,H,seed,lam", [("small", 2, 200, 150, 1, 0.0), ("small", 1, 333, 257, 2, 0.1),
                                                      ("small", 2, 40, 24, 3, 0.0), ("tiny", 3, 64, 48, 0, 0.1)])
def test_pair_adjoint_matches_warp_filter_adjoint(kind, n_cams, W, H, seed, lam):
    sc = S.scene_small(seed=seed) if kind == "small" else S.scene_tiny(seed=seed)
    cams = S.ring_cameras(n_cams, 3.0, W, H, fovx_deg=50.0, phase=0.4 * seed)
    (d0, s0, r0), *others = _adjoint_both(sc, cams, lam)
    assert np.abs(d0).max() > 0
    for d1, s1, r1 in others:
        _close_sums(d1, d0, "dvox")
        if r0 is not None:
            _close_sums(r1, r0, "drgbs")
        assert abs(s1 - s0) <= 1e-4 * abs(s0) + 1e-9   # per-CTA sums agree; CTA atomics in any order


@pytest.mark.parametrize("kind,n_cams,W,H,seed,lam", [("small", 2, 200, 150, 4, 0.0), ("tiny", 3, 64, 48, 1, 0.1),
                                                      ("small", 1, 333, 257, 5, 0.1)])
def test_adjoint_reads_forward_candidate_rows(kind, n_cams, W, H, seed, lam):
    """The CTA-wide adjoint after a CTA-wide forward reads the forward's candidate rows; after a
    forward of another family (no rows) it filters the records itself.  Both give the same
    gradients up to the order of float atomics, and the rows' state follows the calls."""
    from svraster_b200.raster import RasterState
    sc = S.scene_small(seed=seed) if kind == "small" else S.scene_tiny(seed=seed)
    cams = S.ring_cameras(n_cams, 3.0, W, H, fovx_deg=50.0, phase=0.7 * seed)
    ts = torch_scene(sc)
    st = RasterState([cam_dict(c) for c in cams], sc.n_vox, torch.device("cuda"))
    st.preprocess(ts["octpath"], ts["centers"], ts["lengths"], ts["is_leaf"])
    st.bin(ts["octpath"])
    assert not st.candidates_valid()                  # a new binning has no rows
    geos = torch.as_tensor(oracle_inputs(sc, cams[0])[0]).cuda()
    rgbs = torch.as_tensor(np.concatenate([oracle_inputs(sc, c)[1] for c in cams], 0)).cuda()
    s_val = torch.tensor([sc.s_val], dtype=torch.float32, device="cuda")
    gr = [upstream_grads(c.height, c.width, seed=30 + i)[0] for i, c in enumerate(cams)]
    cat = lambda k: torch.as_tensor(np.concatenate([g[k].reshape(-1) for g in gr])).cuda().float()
    L = _lib.load()
    saved = _impl()
    outs = []
    try:
        for fwd_impl, rows in ((3, True), (2, False), (3, True)):
            assert L.svr_render_set_impl(fwd_impl, 3) == 0
            color, depth, normal, T, _ = st.render(3, True, True, ts["centers"], ts["lengths"], geos, rgbs, s_val,
                                                   rgb_per_view=len(cams) > 1)
            assert st.candidates_valid() == rows
            drgbs = torch.zeros(len(cams) * sc.n_vox, 3, device="cuda") if len(cams) > 1 else None
            dvox, ds = st.render_backward(True, True, s_val, T, cat("color"), cat("depth"), cat("normal"), cat("T"),
                                          lambda_R_concen=lam, gt_color=cat("gt") if lam > 0 else None, drgbs=drgbs)
            torch.cuda.synchronize()
            assert st.status() == 0
            outs.append((color.cpu().numpy(), dvox.cpu().numpy(), float(ds.item()),
                         None if drgbs is None else drgbs.cpu().numpy()))
    finally:
        L.svr_render_set_impl(*saved)
    (c0, d0, s0, r0) = outs[0]
    assert np.abs(d0).max() > 0
    for c1, d1, s1, r1 in outs[1:]:
        assert np.array_equal(c1, c0)
        _close_sums(d1, d0, "dvox")
        if r0 is not None:
            _close_sums(r1, r0, "drgbs")
        assert abs(s1 - s0) <= 1e-4 * abs(s0) + 1e-9
    # binning again drops the rows
    st.bin(ts["octpath"])
    assert not st.candidates_valid()
