"""Precision of the GPU render path against the FP64 per-ray oracle, for SH coefficients
stored in f32 and in bf16.

Both paths keep compositing, transmittance and every gradient in f32; only the storage of
the SH coefficients differs.  On random rays of every view (4096 per view) the test compares
colour, transmittance, depth (mean and median), normal and the gradients of the corner SDF
values, per-view colours, SH coefficients and s against the C oracle evaluated in double
precision (libsvr_oracle64, restricted to the sampled pixels).  The bf16 path is compared with
the FP64 oracle given the same bf16 values (arithmetic error) and given the f32 values
(arithmetic + storage error).

Default scale: the precision configuration's scene (the mid-size procedure at levels 6-11,
7.9M voxels) and resolution (1920x1080), on 8 of its 32 views (about 3.4 s of oracle binning
per view); SVR_PRECISION_VIEWS=32 runs all of them.  SVR_PRECISION_SMALL=1 runs the mid-size
scene with 4 views of 960x540 instead.  SVR_PRECISION_OUT=<path> writes the error table as
JSON.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest
import torch

from svraster_b200 import _lib
from svraster_b200 import synthetic as S
from svraster_b200._lib import check, ptr, stream_ptr
from svraster_b200.raster import RasterState

pytestmark = pytest.mark.gpu

FULL = os.environ.get("SVR_PRECISION_SMALL") != "1"
RAYS_PER_VIEW = 4096

# real spherical-harmonics constants of sh_compute.cu (degree 0-3)
C0, C1 = 0.28209479177387814, 0.4886025119029199
C2 = (1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396)
C3 = (-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
      1.445305721320277, -0.5900435899266435)


def sh_basis64(d):
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
    return np.stack([np.full_like(x, C0), -C1 * y, C1 * z, -C1 * x,
                     C2[0] * xy, C2[1] * yz, C2[2] * (2 * zz - xx - yy), C2[3] * xz, C2[4] * (xx - yy),
                     C3[0] * y * (3 * xx - yy), C3[1] * xy * z, C3[2] * y * (4 * zz - xx - yy),
                     C3[3] * z * (2 * zz - 3 * xx - 3 * yy), C3[4] * x * (4 * zz - xx - yy), C3[5] * z * (xx - yy),
                     C3[6] * x * (xx - 3 * yy)], 1)


def _dirs(centers, cam_pos):
    d = centers - cam_pos
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def sh_eval64(centers, cam_pos, sh0, shs, chunk=1 << 20):
    """max(0, sum_k B_k(dir) c_k + 0.5) in double precision."""
    out = np.empty((len(centers), 3))
    for s in range(0, len(centers), chunk):
        e = s + chunk
        B = sh_basis64(_dirs(centers[s:e], cam_pos))
        out[s:e] = B[:, 0:1] * sh0[s:e] + np.einsum("nk,nkc->nc", B[:, 1:], shs[s:e]) + 0.5
    return np.maximum(out, 0.0)


def sh_bw64(centers, cam_positions, drgbs, rows):
    """Coefficient gradients (clamp not differentiated, as the reference) for voxel rows."""
    dsh = np.zeros((len(rows), 16, 3))
    for cp, d in zip(cam_positions, drgbs):
        B = sh_basis64(_dirs(centers[rows], cp))
        dsh += B[:, :, None] * d[rows][:, None, :]
    return dsh


def workload():
    if FULL:
        sc = S.scene_precision(seed=0)
        cams = S.fibonacci_cameras(32, 3.0, 1920, 1080, fovx_deg=50.0)
        cams = cams[:int(os.environ.get("SVR_PRECISION_VIEWS", "8"))]
    else:
        sc = S.scene_mid(seed=0)
        cams = S.fibonacci_cameras(4, 3.0, 960, 540, fovx_deg=50.0)
    return sc, cams


def gpu_pass(sc, cams, t, sh_bf16, grads):
    L = _lib.load()
    dev = t["dev"]
    st = stream_ptr(dev)
    N, V = sc.n_vox, len(cams)
    geos = torch.empty(N, 8, device=dev)
    idx = torch.arange(N, dtype=torch.int64, device=dev)
    check(L.svr_gather_geo(N, ptr(idx), ptr(t["vox_key"]), ptr(t["grid"]), ptr(geos), st), "gather")
    rgbs = torch.empty(V * N, 3, device=dev)
    if sh_bf16:
        sh0, shs = t["sh0"].to(torch.bfloat16).contiguous(), t["shs"].to(torch.bfloat16).contiguous()
        check(L.svr_sh_eval_views_bf16(N, V, 3, 16, ptr(t["centers"]), ptr(t["cam_pos"]), ptr(sh0), ptr(shs),
                                       ptr(rgbs), st), "sh bf16")
    else:
        sh0, shs = t["sh0"], t["shs"]
        check(L.svr_sh_eval_views(N, V, 3, 16, ptr(t["centers"]), ptr(t["cam_pos"]), ptr(sh0), ptr(shs),
                                  ptr(rgbs), st), "sh")
    state = RasterState(t["views"], N, dev)
    state.preprocess(t["octpath"], t["centers"], t["lengths"], t["is_leaf"])
    state.bin(t["octpath"])
    color, depth, normal, T, _ = state.render(3, True, True, t["centers"], t["lengths"], geos, rgbs, t["s_val"],
                                              rgb_per_view=True)
    dvox = torch.zeros(N, 12, device=dev)
    drgbs = torch.zeros(V * N, 3, device=dev)
    ds = torch.zeros(1, device=dev)
    g = {k: torch.as_tensor(v).to(dev) for k, v in grads.items()}
    state.render_backward(True, True, t["s_val"], T, g["color"], g["depth"], g["normal"], g["T"], drgbs=drgbs,
                          dvox=dvox, ds=ds)
    dsh0 = torch.zeros(N, 3, device=dev)
    dshs = torch.zeros(N, 15, 3, device=dev)
    check(L.svr_sh_eval_views_bw(N, V, 3, 16, ptr(t["centers"]), ptr(t["cam_pos"]), ptr(drgbs), ptr(dsh0),
                                 ptr(dshs), st), "sh bw")
    torch.cuda.synchronize()
    assert state.status() == 0
    out = dict(color=color, depth=depth, normal=normal, T=T, dvox=dvox, drgbs=drgbs.view(V, N, 3), ds=ds,
               dsh=torch.cat([dsh0[:, None], dshs], 1))
    return {k: v.cpu().numpy().astype(np.float64) for k, v in out.items()}


def oracle_pass(sc, cams, rays, grads_v, sh_sets, geos64):
    """FP64 per-ray oracle on the sampled pixels of every view, once per SH coefficient set
    (binning is shared: it does not depend on the colours)."""
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    N = sc.n_vox
    centers64 = sc.vox_center.astype(np.float64)
    out = [dict(img=[], dvox=np.zeros((N, 12)), drgbs=[], ds=0.0) for _ in sh_sets]
    for v, cam in enumerate(cams):
        H, W = cam.height, cam.width
        mask = np.zeros(H * W, np.uint8)
        mask[rays[v]] = 1
        nd, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
        _, vals, ranges = O.binning(cam, sc.octpath, nd, bb, bits)
        for res, (sh0, shs) in zip(out, sh_sets):
            rgbs = sh_eval64(centers64, cam.position.astype(np.float64), sh0, shs)
            O.set_pixel_mask(mask, bits=64)
            try:
                bg = np.zeros(3, np.float32)
                f = O.render_fwd(cam, bg, 3, True, True, ranges, vals, bb, sc.vox_center, sc.vox_size, geos64,
                                 rgbs, sc.s_val, bits=64)
                g = grads_v[v]
                dvox, ds = O.render_bwd(cam, bg, True, True, ranges, f["tile_last"], vals, bb, sc.vox_center,
                                        sc.vox_size, geos64, rgbs, sc.s_val, f["T"], f["n_contrib"], g["color"],
                                        g["depth"], g["normal"], g["T"], bits=64)
            finally:
                O.set_pixel_mask(None, bits=64)
            res["img"].append(f)
            res["dvox"][:, :8] += dvox[:, :8]
            res["dvox"][:, 11] += dvox[:, 11]
            res["drgbs"].append(dvox[:, 8:11].copy())
            res["ds"] += ds
    for res in out:
        rows = np.nonzero(np.any([np.any(d != 0, axis=1) for d in res["drgbs"]], axis=0))[0]
        res["dsh_rows"] = rows
        res["dsh"] = sh_bw64(centers64, [c.position.astype(np.float64) for c in cams], res["drgbs"], rows)
    return out


def _img_errors(gpu, ref, cams, rays):
    err = {k: [] for k in ("color", "T", "depth_mean", "depth_median", "normal")}
    off = 0
    for v, cam in enumerate(cams):
        P = cam.width * cam.height
        r = rays[v]
        f = ref["img"][v]
        g_color = gpu["color"][3 * off:3 * (off + P)].reshape(3, P)
        g_depth = gpu["depth"][4 * off:4 * (off + P)].reshape(4, P)
        g_normal = gpu["normal"][3 * off:3 * (off + P)].reshape(3, P)
        g_T = gpu["T"][off:off + P]
        err["color"].append(np.abs(g_color[:, r] - f["color"].reshape(3, P)[:, r]).ravel())
        err["T"].append(np.abs(g_T[r] - f["T"].reshape(P)[r]))
        err["depth_mean"].append(np.abs(g_depth[0, r] - f["depth"].reshape(4, P)[0, r]))
        err["depth_median"].append(np.abs(g_depth[2, r] - f["depth"].reshape(4, P)[2, r]))
        err["normal"].append(np.abs(g_normal[:, r] - f["normal"].reshape(3, P)[:, r]).ravel())
        off += P
    out = {}
    for k, e in err.items():
        e = np.concatenate(e)
        out[k] = dict(max=float(e.max()), p999=float(np.quantile(e, 0.999)), mean=float(e.mean()),
                      frac_above_1e3=float((e > 1e-3).mean()))
    return out


def _rel(a, b):
    """|a - b| / max|b| over entries: max and 99.9th percentile."""
    scale = float(np.abs(b).max())
    e = np.abs(a - b) / max(scale, 1e-30)
    return dict(max=float(e.max()), p999=float(np.quantile(e, 0.999)), scale=scale)


def _grad_errors(gpu, ref):
    rows = ref["dsh_rows"]
    return {"corner_sdf": _rel(gpu["dvox"][:, :8], ref["dvox"][:, :8]),
            "abs_dalpha_alpha": _rel(gpu["dvox"][:, 11], ref["dvox"][:, 11]),
            "view_rgb": _rel(gpu["drgbs"], np.stack(ref["drgbs"])),
            "sh_coefficients": _rel(gpu["dsh"][rows], ref["dsh"]),
            "s": dict(rel=float(abs(gpu["ds"][0] - ref["ds"]) / max(abs(ref["ds"]), 1e-30)))}


def test_precision_against_fp64_oracle():
    dev = torch.device("cuda")
    sc, cams = workload()
    rng = np.random.default_rng(0)
    rays = [rng.choice(c.width * c.height, RAYS_PER_VIEW, replace=False) for c in cams]
    # upstream gradients: N(0,1) on the sampled rays only (colour, mean depth, normal)
    grads_v = []
    for v, cam in enumerate(cams):
        P = cam.width * cam.height
        gc = np.zeros((3, P), np.float32)
        gd = np.zeros((4, P), np.float32)
        gn = np.zeros((3, P), np.float32)
        gc[:, rays[v]] = rng.normal(size=(3, RAYS_PER_VIEW))
        gd[0, rays[v]] = rng.normal(size=RAYS_PER_VIEW)
        gn[:, rays[v]] = rng.normal(size=(3, RAYS_PER_VIEW))
        grads_v.append(dict(color=gc, depth=gd, normal=gn, T=np.zeros(P, np.float32)))
    # per-view planes are packed view after view ([ch, P_v] blocks)
    packed = {k: np.concatenate([g[k].reshape(-1) for g in grads_v]).astype(np.float32)
              for k in ("color", "depth", "normal", "T")}
    f32 = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    t = dict(dev=dev, octpath=f32(sc.octpath, torch.int64), centers=f32(sc.vox_center),
             lengths=f32(sc.vox_size).reshape(-1).contiguous(), is_leaf=f32(sc.is_leaf, torch.uint8),
             vox_key=f32(sc.vox_key, torch.int64), grid=f32(sc.geo_grid_pts), sh0=f32(sc.sh0), shs=f32(sc.shs),
             s_val=torch.tensor([sc.s_val], dtype=torch.float32, device=dev),
             cam_pos=torch.stack([f32(c.c2w)[:3, 3] for c in cams]).contiguous())
    t["views"] = [dict(width=c.width, height=c.height, tanfovx=c.tanfovx, tanfovy=c.tanfovy, cx=c.cx, cy=c.cy,
                       near=c.near, w2c=f32(c.w2c), c2w=f32(c.c2w), bg=torch.zeros(3, device=dev)) for c in cams]

    gpu32 = gpu_pass(sc, cams, t, False, packed)
    gpu16 = gpu_pass(sc, cams, t, True, packed)
    del t
    torch.cuda.empty_cache()

    geos64 = sc.geo_grid_pts.reshape(-1).astype(np.float64)[sc.vox_key]
    sh0_32, shs_32 = sc.sh0.astype(np.float64), sc.shs.astype(np.float64)
    bf = lambda a: torch.as_tensor(a).to(torch.bfloat16).to(torch.float64).numpy()
    sh0_16, shs_16 = bf(sc.sh0), bf(sc.shs)
    ref32, ref16 = oracle_pass(sc, cams, rays, grads_v, [(sh0_32, shs_32), (sh0_16, shs_16)], geos64)

    report = {
        "workload": ("precision: 3 spheres + torus, levels 6-11" if FULL else "mid-size: 3 spheres + torus, levels 6-10")
                    + f", {sc.n_vox} voxels, {len(cams)} views {cams[0].width}x{cams[0].height}, "
                      f"{RAYS_PER_VIEW} random rays per view",
        "f32_sh_vs_fp64": {"images": _img_errors(gpu32, ref32, cams, rays), "gradients": _grad_errors(gpu32, ref32)},
        "bf16_sh_vs_fp64_same_bf16_values": {"images": _img_errors(gpu16, ref16, cams, rays),
                                             "gradients": _grad_errors(gpu16, ref16)},
        "bf16_sh_vs_fp64_f32_values": {"images": _img_errors(gpu16, ref32, cams, rays),
                                       "gradients": _grad_errors(gpu16, ref32)},
    }
    print("PRECISION", json.dumps(report))
    if os.environ.get("SVR_PRECISION_OUT"):
        with open(os.environ["SVR_PRECISION_OUT"], "w") as fh:
            json.dump(report, fh, indent=1)

    # images within 1e-3 of the FP64 oracle (a few rays may end one record apart at the
    # early-termination threshold), gradients within 1e-3 of the largest entry
    for key in ("f32_sh_vs_fp64", "bf16_sh_vs_fp64_same_bf16_values"):
        im, gr = report[key]["images"], report[key]["gradients"]
        for k in ("color", "T", "normal"):
            assert im[k]["p999"] < 1e-3 and im[k]["frac_above_1e3"] < 2e-3, (key, k, im[k])
        for k in ("depth_mean", "depth_median"):
            assert im[k]["p999"] < 3e-3, (key, k, im[k])
        for k in ("corner_sdf", "view_rgb", "sh_coefficients"):
            assert gr[k]["p999"] < 1e-3, (key, k, gr[k])
    # storage rounding of the coefficients: colour error bounded by the bf16 step
    assert report["bf16_sh_vs_fp64_f32_values"]["images"]["color"]["max"] < 2e-2
