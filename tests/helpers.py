"""Shared fixtures of the parity tests: seeded scenes, cameras, and both implementations
(the sm_100a library through the C ABI, the C oracle) run on the same inputs."""
from __future__ import annotations

import numpy as np

from svraster_b200 import synthetic as S


def scene_and_cams(kind="tiny", n_cams=2, W=128, H=96, seed=0):
    if kind == "tiny":
        sc = S.scene_tiny(seed=seed)
    elif kind == "small":
        sc = S.scene_small(seed=seed)
    else:
        raise ValueError(kind)
    cams = S.ring_cameras(n_cams, 3.0, W, H, fovx_deg=50.0, phase=0.3 + seed)
    return sc, cams


def oracle_inputs(sc, cam):
    """geos / rgbs from the oracle's gather and SH (these are exactly reproducible)."""
    from oracle import oracle as O
    geos = O.gather_geo(np.arange(sc.n_vox), sc.vox_key, sc.geo_grid_pts, sc.n_vox)
    rgbs = O.sh_eval(3, None, sc.vox_center, cam.position, sc.sh0, sc.shs)
    return geos, rgbs


def upstream_grads(H, W, seed=1, n_views=1):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_views):
        out.append(dict(color=rng.normal(size=(3, H, W)).astype(np.float32),
                        depth=rng.normal(size=(4, H, W)).astype(np.float32),
                        normal=rng.normal(size=(3, H, W)).astype(np.float32),
                        T=rng.normal(size=(1, H, W)).astype(np.float32) * 0.1,
                        gt=rng.uniform(size=(3, H, W)).astype(np.float32)))
    return out


def oracle_view(sc, cam, geos, rgbs, n_samp=3, need_depth=True, need_normal=True, grads=None, lambda_R=0.0,
                bg=(0.0, 0.0, 0.0)):
    from oracle import oracle as O
    bg = np.asarray(bg, np.float32)
    nd, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
    keys, vals, ranges = O.binning(cam, sc.octpath, nd, bb, bits)
    tr = np.zeros(cam.width * cam.height, np.uint8)
    O.set_trace(tr)
    try:
        f = O.render_fwd(cam, bg, n_samp, need_depth, need_normal, ranges, vals, bb, sc.vox_center, sc.vox_size,
                         geos, rgbs, sc.s_val, track_max_w=True)
    finally:
        O.set_trace(None)
    res = dict(n_dup=nd, bbox=bb, bits=bits, keys=keys, vals=vals, ranges=ranges, flags=forward_flags(cam, tr), **f)
    if grads is not None:
        dvox, ds = O.render_bwd(cam, bg, need_depth, need_normal, ranges, f["tile_last"], vals, bb, sc.vox_center,
                                sc.vox_size, geos, rgbs, sc.s_val, f["T"], f["n_contrib"], grads["color"],
                                grads["depth"], grads["normal"], grads["T"], lambda_R, grads["gt"])
        res["dvox"], res["ds"] = dvox, ds
    return res


def assert_close(name, got, ref, rtol, atol, max_bad_frac=0.0):
    got = np.asarray(got, np.float64); ref = np.asarray(ref, np.float64)
    assert got.shape == ref.shape, f"{name}: shape {got.shape} vs {ref.shape}"
    err = np.abs(got - ref)
    bad = err > atol + rtol * np.abs(ref)
    frac = bad.mean() if bad.size else 0.0
    worst = float(err.max()) if err.size else 0.0
    assert frac <= max_bad_frac, (f"{name}: {bad.sum()} / {bad.size} elements out of tolerance "
                                  f"(max abs err {worst:.3e}, rtol {rtol}, atol {atol})")
    return worst


def torch_scene(sc, device="cuda"):
    import torch
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(device, dt)
    return dict(octpath=t(sc.octpath, torch.int64), centers=t(sc.vox_center), lengths=t(sc.vox_size).reshape(-1),
                is_leaf=t(sc.is_leaf, torch.uint8), vox_key=t(sc.vox_key, torch.int64), grid=t(sc.geo_grid_pts),
                sh0=t(sc.sh0), shs=t(sc.shs))


def cam_dict(cam, bg=(0.0, 0.0, 0.0), device="cuda"):
    import torch
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(device)
    return dict(width=cam.width, height=cam.height, tanfovx=cam.tanfovx, tanfovy=cam.tanfovy, cx=cam.cx,
                cy=cam.cy, near=cam.near, w2c=t(cam.w2c), c2w=t(cam.c2w), bg=t(bg))


def cuda_views(sc, cams, geos_list, rgbs_list, n_samp=3, need_depth=True, need_normal=True, grads_list=None,
               lambda_R=0.0, bg=(0.0, 0.0, 0.0), track_max_w=False):
    """Render a batch of views through the C ABI; geos shared, rgbs per view."""
    import torch
    from svraster_b200.raster import RasterState
    ts = torch_scene(sc)
    views = [cam_dict(c, bg) for c in cams]
    st = RasterState(views, sc.n_vox, torch.device("cuda"))
    n_dup = st.preprocess(ts["octpath"], ts["centers"], ts["lengths"], ts["is_leaf"])
    st.bin(ts["octpath"])
    geos = torch.as_tensor(geos_list).cuda().float().contiguous()
    rgbs = torch.as_tensor(np.concatenate(rgbs_list, 0)).cuda().float().contiguous()
    s_val = torch.tensor([sc.s_val], dtype=torch.float32, device="cuda")
    color, depth, normal, T, max_w = st.render(n_samp, need_depth, need_normal, ts["centers"], ts["lengths"], geos,
                                               rgbs, s_val, track_max_w=track_max_w, rgb_per_view=len(cams) > 1)
    out = dict(state=st, n_dup=n_dup, color=color, depth=depth, normal=normal, T=T, max_w=max_w)
    if grads_list is not None:
        cat = lambda k: torch.as_tensor(np.concatenate([g[k].reshape(-1) for g in grads_list])).cuda().float()
        drgbs = torch.zeros(len(cams) * sc.n_vox, 3, device="cuda") if len(cams) > 1 else None
        dvox, ds = st.render_backward(need_depth, need_normal, s_val, T, cat("color"), cat("depth"), cat("normal"),
                                      cat("T"), lambda_R_concen=lambda_R, gt_color=cat("gt") if lambda_R > 0 else None,
                                      drgbs=drgbs)
        out["dvox"], out["ds"], out["drgbs"] = dvox, ds, drgbs
    torch.cuda.synchronize()
    return out


def split_view(arr, views, v, channels):
    """Slice view v's planes out of a packed per-view output."""
    off = sum(c.width * c.height for c in views[:v])
    n = views[v].width * views[v].height
    a = arr.reshape(-1)[channels * off: channels * (off + n)]
    return a.reshape(channels, views[v].height, views[v].width)


# Image parity on the pixels whose forward decisions are not at a threshold (the oracle's
# trace: alpha within ulps of MIN_ALPHA, T at the early stop or a median-depth decision at
# T = 0.5): |got - ref| <= 1e-5 of the channel's range everywhere, and <= 1e-5 of |ref| for all
# but 0.2% of the entries above 1% of the range (float32 evaluations of the same expressions;
# the device's expf and the host's differ by an ulp, alpha = (phi_e - phi_x) / phi_e cancels).
IMG_RANGE_TOL, IMG_ELEM_TOL, IMG_ELEM_FRAC = 1e-5, 1e-5, 2e-3
FLIP_FWD = 1 | 2 | 4


def image_parity(got, ref, flagged):
    """Errors of one plane group [C, ...] on the unflagged pixels: relative to each channel's
    range, and per element for entries at least 1% of the range."""
    got = np.asarray(got, np.float64).reshape(np.shape(ref)[0], -1)
    ref = np.asarray(ref, np.float64).reshape(np.shape(ref)[0], -1)
    ok = ~np.asarray(flagged).reshape(-1)
    rng = np.abs(ref).max(axis=1, keepdims=True) + 1e-30
    err = np.abs(got - ref)[:, ok]
    r_range = err / rng
    big = (np.abs(ref) >= 1e-2 * rng)[:, ok]
    r_elem = (err / (np.abs(ref[:, ok]) + 1e-30))[big]
    return {"range_rel_max": float(r_range.max()) if r_range.size else 0.0,
            "elem_rel_max": float(r_elem.max()) if r_elem.size else 0.0,
            "elem_rel_p999": float(np.quantile(r_elem, 0.999)) if r_elem.size else 0.0,
            "elem_over_tol": int((r_elem > IMG_ELEM_TOL).sum()), "elements": int(r_elem.size),
            "bitwise_equal_frac": float((got[:, ok] == ref[:, ok]).mean()) if ok.any() else 1.0}


def assert_image_parity(tag, stats):
    assert stats["range_rel_max"] <= IMG_RANGE_TOL, (tag, stats)
    assert stats["elem_over_tol"] <= IMG_ELEM_FRAC * max(stats["elements"], 1), (tag, stats)


def images_match(got, ref, flagged, tag=""):
    """Colour, depth, normal and T of one view against a reference render ({name: [C,H,W]})."""
    out = {}
    for key in ("color", "depth", "normal", "T"):
        if key in got and got[key] is not None:
            out[key] = image_parity(got[key], ref[key], flagged)
            assert_image_parity(f"{tag} {key}", out[key])
    return out


def forward_flags(cam, trace):
    """Pixels [H, W] with a forward decision at a threshold, from an oracle pixel trace."""
    return ((np.asarray(trace) & FLIP_FWD) > 0).reshape(cam.height, cam.width)
