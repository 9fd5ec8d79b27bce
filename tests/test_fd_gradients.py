"""Gradient checks of the adjoint against FP64 central finite differences.

The FP64 per-ray oracle (oracle/libsvr_oracle64.so: the reference algorithm evaluated in
double) renders a small scene; the loss is the inner product of the outputs with fixed
upstream gradients.  Central differences over randomly chosen corner SDFs and colours are
compared with the oracle's adjoint (the reference's backward formulas in double), and the
sm_100a library's float32 adjoint is compared with the same FP64 gradients.
"""
import numpy as np
import pytest

from svraster_b200 import synthetic as S
from tests.helpers import oracle_inputs


def _setup(seed=0, W=40, H=32):
    from oracle import oracle as O
    sc = S.scene_tiny(seed=seed)
    cam = S.ring_cameras(1, 3.0, W, H, phase=0.4 + seed)[0]
    geos32, rgbs32 = oracle_inputs(sc, cam)
    nd, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
    keys, vals, ranges = O.binning(cam, sc.octpath, nd, bb, bits)
    rng = np.random.default_rng(seed + 100)
    up = dict(color=rng.normal(size=(3, H, W)), depth=rng.normal(size=(4, H, W)), normal=rng.normal(size=(3, H, W)))
    up["depth"][1:] = 0.0     # only the mean-depth channel is differentiated (backward.cu:180)
    return sc, cam, geos32.astype(np.float64), rgbs32.astype(np.float64), vals, ranges, bb, up


def _loss(O, sc, cam, geos, rgbs, vals, ranges, bb, up):
    f = O.render_fwd(cam, np.zeros(3, np.float32), 3, True, True, ranges, vals, bb, sc.vox_center.astype(np.float64),
                     sc.vox_size.astype(np.float64), geos, rgbs, sc.s_val, bits=64)
    L = (f["color"] * up["color"]).sum() + (f["depth"] * up["depth"]).sum() + (f["normal"] * up["normal"]).sum()
    return L, f


def test_fp64_adjoint_matches_central_differences():
    from oracle import oracle as O
    sc, cam, geos, rgbs, vals, ranges, bb, up = _setup()
    L0, f = _loss(O, sc, cam, geos, rgbs, vals, ranges, bb, up)
    dvox, _ = O.render_bwd(cam, np.zeros(3, np.float32), True, True, ranges, f["tile_last"], vals, bb,
                           sc.vox_center.astype(np.float64), sc.vox_size.astype(np.float64), geos, rgbs, sc.s_val,
                           f["T"], f["n_contrib"], up["color"], up["depth"], up["normal"],
                           np.zeros((1, cam.height, cam.width)), bits=64)
    rng = np.random.default_rng(7)
    touched = np.where(np.abs(dvox).sum(1) > 0)[0]
    pick = rng.choice(touched, size=min(150, len(touched)), replace=False)
    errs = []
    for i in pick:
        for which in ("geo", "rgb"):
            k = rng.integers(0, 8 if which == "geo" else 3)
            arr = geos if which == "geo" else rgbs
            h = 1e-7 * max(1.0, abs(arr[i, k]))
            old = arr[i, k]
            arr[i, k] = old + h
            Lp, _ = _loss(O, sc, cam, geos, rgbs, vals, ranges, bb, up)
            arr[i, k] = old - h
            Lm, _ = _loss(O, sc, cam, geos, rgbs, vals, ranges, bb, up)
            arr[i, k] = old
            fd = (Lp - Lm) / (2 * h)
            an = dvox[i, k] if which == "geo" else dvox[i, 8 + k]
            errs.append(abs(fd - an) / max(abs(fd), abs(an), 1e-3))
    errs = np.array(errs)
    # kinks (alpha clamp / early stop / median selection) may land inside a step: allow a few
    assert np.median(errs) < 1e-6, np.median(errs)
    assert np.quantile(errs, 0.95) < 1e-4, np.quantile(errs, 0.95)


@pytest.mark.gpu
def test_library_adjoint_matches_fp64_oracle():
    from oracle import oracle as O
    from tests.helpers import cuda_views
    sc, cam, geos, rgbs, vals, ranges, bb, up = _setup(seed=1, W=96, H=80)
    L0, f = _loss(O, sc, cam, geos, rgbs, vals, ranges, bb, up)
    ref, _ = O.render_bwd(cam, np.zeros(3, np.float32), True, True, ranges, f["tile_last"], vals, bb,
                          sc.vox_center.astype(np.float64), sc.vox_size.astype(np.float64), geos, rgbs, sc.s_val,
                          f["T"], f["n_contrib"], up["color"], up["depth"], up["normal"],
                          np.zeros((1, cam.height, cam.width)), bits=64)
    grads = dict(color=up["color"].astype(np.float32), depth=up["depth"].astype(np.float32),
                 normal=up["normal"].astype(np.float32), T=np.zeros((1, cam.height, cam.width), np.float32),
                 gt=np.zeros((3, cam.height, cam.width), np.float32))
    out = cuda_views(sc, [cam], geos.astype(np.float32), [rgbs.astype(np.float32)], grads_list=[grads])
    got = out["dvox"].cpu().numpy().astype(np.float64)
    col_scale = np.abs(ref).max(0) + 1e-12
    err = np.abs(got - ref) / col_scale
    assert np.quantile(err, 0.999) < 1e-3
    # image against the FP64 oracle (north-star bound 1e-3)
    img = out["color"].cpu().numpy().reshape(3, cam.height, cam.width)
    assert np.abs(img - f["color"]).max() < 1e-3
