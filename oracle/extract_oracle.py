"""NumPy restatement of the reference's TSDF fusion and marching cubes -- TEST INFRASTRUCTURE.

* ``tsdf_integrate`` follows src/utils/fuser_utils.py:54-148 (Fuser.integrate) with the
  projection of src/cameras.py:89-103 and torch's bilinear grid_sample (zeros padding,
  align_corners=False), one float32 operation at a time.
* ``marching_cubes`` follows cuda/svraster_cuda/marching_cubes.py:271-380.  The case table is
  read from the library's packed copy (svraster_b200/csrc/mc_table.inc); both are pinned to
  the reference by the golden fixtures.
Pinned against tests/golden/extract_*.npz (the reference's own torch code run on CPU).
"""
from __future__ import annotations

import os
import re

import numpy as np

F = np.float32
_HERE = os.path.dirname(os.path.abspath(__file__))


def _bilinear(img, u, v):
    H, W = img.shape
    ix = ((u + F(1)) * F(W) - F(1)) / F(2)
    iy = ((v + F(1)) * F(H) - F(1)) / F(2)
    ix_nw = np.floor(ix).astype(np.int64)
    iy_nw = np.floor(iy).astype(np.int64)
    out = np.zeros_like(u)
    for dx, dy in ((0, 0), (1, 0), (0, 1), (1, 1)):
        xx, yy = ix_nw + dx, iy_nw + dy
        wx = (ix - xx.astype(F)) if dx == 0 else (xx.astype(F) - ix)
        wy = (iy - yy.astype(F)) if dy == 0 else (yy.astype(F) - iy)
        # weight of corner (dx, dy) is the product of the distances to the opposite corner
        wgt = ((ix_nw + 1 - dx).astype(F) - ix) * ((iy_nw + 1 - dy).astype(F) - iy) if (dx, dy) == (0, 0) else None
        ok = (xx >= 0) & (xx < W) & (yy >= 0) & (yy < H)
        if dx == 0 and dy == 0:
            w = ((ix_nw + 1).astype(F) - ix) * ((iy_nw + 1).astype(F) - iy)
        elif dx == 1 and dy == 0:
            w = (ix - ix_nw.astype(F)) * ((iy_nw + 1).astype(F) - iy)
        elif dx == 0 and dy == 1:
            w = ((ix_nw + 1).astype(F) - ix) * (iy - iy_nw.astype(F))
        else:
            w = (ix - ix_nw.astype(F)) * (iy - iy_nw.astype(F))
        val = np.zeros_like(u)
        val[ok] = img[yy[ok], xx[ok]]
        out = out + val * w
    return out


def tsdf_integrate(weight, sd_val, xyz, w2c, c2w, tanfovx, tanfovy, cx_p, cy_p, depth, alpha, bandwidth,
                   use_trunc=True, alpha_thres=0.5, crop_border=0.0, depth_weight=False, border_weight=False,
                   max_norm_dist=10.0):
    """One view of fuser_utils.py:54-148; updates weight / sd_val [M,1] in place."""
    p = xyz.astype(F)
    R = w2c[:3, :3].astype(F)
    t = w2c[:3, 3].astype(F)
    cam = p[:, [0]] * R[:, 0] + p[:, [1]] * R[:, 1] + p[:, [2]] * R[:, 2] + t
    uv = cam[:, :2] / cam[:, [2]]
    uv[:, 0] = uv[:, 0] * F(1 / tanfovx) + F(2 * cx_p - 1)
    uv[:, 1] = uv[:, 1] * F(1 / tanfovy) + F(2 * cy_p - 1)
    keep = np.where((np.abs(uv) <= F(1 - crop_border)).all(-1))[0]
    u, v = uv[keep, 0], uv[keep, 1]
    d = _bilinear(depth.reshape(depth.shape[-2:]).astype(F), u, v)
    pos = c2w[:3, 3].astype(F)
    look = c2w[:3, 2].astype(F)
    q = p[keep] - pos
    xyz_depth = q[:, 0] * look[0] + q[:, 1] * look[1] + q[:, 2] * look[2]
    sdf = d - xyz_depth
    inv = (F(1) / bandwidth[keep].astype(F)) if isinstance(bandwidth, np.ndarray) else F(1 / bandwidth)
    sdf = sdf * inv
    idx = keep
    if use_trunc:
        sel = np.where(sdf >= F(-1))[0]
        idx, u, v, d, sdf = idx[sel], u[sel], v[sel], d[sel], np.clip(sdf[sel], F(-1), F(1))
        w = np.ones_like(d)
    else:
        w = np.exp(-np.minimum(np.abs(sdf), F(max_norm_dist))).astype(F)
    if alpha is not None:
        a = _bilinear(alpha.reshape(alpha.shape[-2:]).astype(F), u, v)
        w = w * a
        sel = np.where(a >= F(alpha_thres))[0]
        idx, u, v, d, sdf, w = idx[sel], u[sel], v[sel], d[sel], sdf[sel], w[sel]
    if depth_weight:
        w = w * (F(1) / np.maximum(d, F(0.1)))
    if border_weight:
        w = w * (F(1) / (F(1) + F(9 / np.sqrt(2)) * np.sqrt(u * u + v * v)))
    weight[idx, 0] = weight[idx, 0] + w
    sd_val[idx, 0] = sd_val[idx, 0] + w * sdf


def _mc_table():
    path = os.path.join(os.path.dirname(_HERE), "svraster_b200", "csrc", "mc_table.inc")
    words = [int(x, 16) for x in re.findall(r"0x([0-9a-f]{16})ull", open(path).read())]
    tab = np.full((256, 15), -1, np.int64)
    for c, w in enumerate(words):
        for k in range(15):
            e = (w >> (4 * k)) & 15
            tab[c, k] = -1 if e == 15 else e
    return tab


_PAIRS = [[0, 1], [1, 5], [5, 4], [4, 0], [2, 3], [3, 7], [7, 6], [6, 2], [0, 2], [1, 3], [5, 7], [4, 6]]


def marching_cubes(val, xyz, vox_key, iso):
    """marching_cubes.py:278-380 -> (verts f32[V,3] sorted unique, faces i64[F,3])."""
    unit_val = val.astype(F)[vox_key]
    unit_xyz = xyz.astype(F)[vox_key]
    m = (unit_val > F(iso)).any(1) & (unit_val < F(iso)).any(1) & ~np.isnan(unit_val).any(1)
    unit_val, unit_xyz = unit_val[m], unit_xyz[m]
    n = len(unit_val)
    if n == 0:
        return np.zeros((0, 3), F), np.zeros((0, 3), np.int64)
    verts = np.zeros((n, 12, 3), F)
    for i, (a, b) in enumerate(_PAIRS):
        v1, v2 = unit_val[:, a], unit_val[:, b]
        with np.errstate(divide="ignore", invalid="ignore"):
            r = (F(iso) - v1) / (v2 - v1)
        r[np.abs(v1 - v2) < F(1e-9)] = F(0.5)
        verts[:, i] = unit_xyz[:, a] + r[:, None] * (unit_xyz[:, b] - unit_xyz[:, a])
    cube = ((unit_val < F(iso)).astype(np.int64) << np.arange(8)).sum(1)
    tri = _mc_table()[cube]
    fx = verts[np.arange(n)[:, None], tri]
    fx = fx[tri != -1]
    uniq, inv = np.unique(fx, axis=0, return_inverse=True)
    return uniq.astype(F), inv.reshape(-1, 3).astype(np.int64)
