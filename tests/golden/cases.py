"""Seeded inputs of the golden-vector cases (shared by the generator and the tests)."""
from __future__ import annotations

import hashlib

import numpy as np

from svraster_b200 import synthetic as S

# vox_geo_mode 3 = triinterp3 (the shipped SDF setting), 1 = triinterp1 (forward only differs)
CASES = {
    "tiny_v0": dict(seed=0, view=0, n_views=2, W=64, H=48, phase=0.3, bg=(0.0, 0.0, 0.0), lambda_R_concen=0.0,
                    vox_geo_mode=3),
    "tiny_v1": dict(seed=0, view=1, n_views=2, W=64, H=48, phase=0.3, bg=(0.1, 0.2, 0.3), lambda_R_concen=0.1,
                    vox_geo_mode=3),
    "tiny_s1": dict(seed=1, view=0, n_views=1, W=80, H=60, phase=1.3, bg=(0.0, 0.0, 0.0), lambda_R_concen=0.0,
                    vox_geo_mode=3),
}
TABLE_CASE = dict(seed=0, res_pow2=5, weight=0.01, vox_size_inv=16.0, drop=0.0)
ADAM_CASE = dict(seed=3, n=4099, step=7, lr=0.01, beta1=0.1, beta2=0.99, eps=1e-15)
# voxel Eikonal, sign total variation and points loss (vg / tv / pl_compute.cu)
REG_CASE = dict(seed=0, res_pow2=5, weight=0.01, n_points=6000)


def digest(inp):
    h = hashlib.sha256()
    for k in sorted(inp):
        v = inp[k]
        if isinstance(v, np.ndarray):
            h.update(k.encode()); h.update(np.ascontiguousarray(v).tobytes())
        elif isinstance(v, S.Scene):
            for f in ("octpath", "vox_center", "vox_size", "is_leaf", "vox_key", "geo_grid_pts", "sh0", "shs"):
                h.update(np.ascontiguousarray(getattr(v, f)).tobytes())
        elif isinstance(v, S.Camera):
            h.update(v.w2c.tobytes()); h.update(v.c2w.tobytes())
        elif isinstance(v, dict):
            for kk in sorted(v):
                h.update(np.ascontiguousarray(v[kk]).tobytes())
    return h.hexdigest()


def build_case_inputs(case):
    sc = S.scene_tiny(seed=case["seed"])
    cams = S.ring_cameras(case["n_views"], 3.0, case["W"], case["H"], fovx_deg=50.0, phase=case["phase"])
    cam = cams[case["view"]]
    rng = np.random.default_rng(100 + case["seed"] * 10 + case["view"])
    H, W = cam.height, cam.width
    grads = dict(color=rng.normal(size=(3, H, W)).astype(np.float32),
                 depth=rng.normal(size=(4, H, W)).astype(np.float32),
                 normal=rng.normal(size=(3, H, W)).astype(np.float32),
                 T=(0.1 * rng.normal(size=(1, H, W))).astype(np.float32),
                 gt=rng.uniform(size=(3, H, W)).astype(np.float32))
    return dict(scene=sc, cam=cam, grads=grads)


def grid_voxel_geometry(sc, res_pow2):
    """grid_voxel_coord / grid_voxel_size as train.py:963-966 computes them."""
    res = float(1 << res_pow2)
    ext = np.float32(sc.scene_extent)
    smin = np.float32(0.0) - ext * np.float32(0.5)
    coord = ((sc.vox_center - sc.vox_size * np.float32(0.5)) - smin) / ext * np.float32(res)
    size = (sc.vox_size / ext) * np.float32(res)
    return np.round(coord).astype(np.float32), np.round(size).astype(np.float32).reshape(-1)


def build_table_inputs(case):
    from oracle import oracle as O
    sc = S.scene_tiny(seed=case["seed"])
    coord, size = grid_voxel_geometry(sc, case["res_pow2"])
    mask, keys, g2v = O.valid_table(sc.vox_center, sc.vox_size, np.zeros(3, np.float32), sc.scene_extent,
                                    case["res_pow2"], sc.is_leaf)
    G = len(keys)
    rng = np.random.default_rng(case["seed"] + 7)
    K = int(G * (1.0 - case["drop"]))
    active = rng.permutation(G)[:K].astype(np.int32)
    return dict(scene=sc, grid_voxel_coord=coord, grid_voxel_size=size, active=active, expected_count=G)


def build_adam_inputs(case):
    rng = np.random.default_rng(case["seed"])
    n = case["n"]
    grad = rng.normal(size=n).astype(np.float32)
    grad[rng.random(n) < 0.2] = 0.0
    return dict(param=rng.normal(size=n).astype(np.float32), grad=grad,
                m=(0.1 * rng.normal(size=n)).astype(np.float32), v=np.abs(0.1 * rng.normal(size=n)).astype(np.float32))


def build_reg_inputs(case):
    """Inputs of the voxel-Eikonal / total-variation / points-loss case: the table case's scene,
    a voxel list with repeats, a 3-channel grid quantised to 1/4 so that neighbours tie, a
    sparse nonzero starting gradient, and points (grid units) both inside masked cells and
    scattered over and beyond the grid."""
    from oracle import oracle as O
    sc = S.scene_tiny(seed=case["seed"])
    rng = np.random.default_rng(case["seed"] + 11)
    N, M = sc.n_vox, sc.geo_grid_pts.shape[0]
    res = 1 << case["res_pow2"]
    coord, size = grid_voxel_geometry(sc, case["res_pow2"])
    mask, keys, g2v = O.valid_table(sc.vox_center, sc.vox_size, np.zeros(3, np.float32), sc.scene_extent,
                                    case["res_pow2"], sc.is_leaf)
    active = rng.integers(0, N, size=int(N * 0.8)).astype(np.int32)
    grid3 = (np.round(rng.normal(size=(M, 3)) * 4.0) / 4.0).astype(np.float32)
    grad1 = np.where(rng.random((M, 1)) < 0.1, rng.normal(size=(M, 1)), 0.0).astype(np.float32)
    grad3 = np.where(rng.random((M, 3)) < 0.1, rng.normal(size=(M, 3)), 0.0).astype(np.float32)
    P = case["n_points"]
    cells = np.flatnonzero(mask)
    pick = cells[rng.integers(0, len(cells), size=P // 2)]
    inside = np.stack([pick % res, (pick // res) % res, pick // (res * res)], 1) + rng.random((P // 2, 3))
    spread = rng.uniform(-2.0, res + 2.0, size=(P - P // 2, 3))
    points = np.concatenate([inside, spread]).astype(np.float32)
    return dict(scene=sc, vox_size_inv=(1.0 / sc.vox_size.reshape(-1)).astype(np.float32), active=active,
                grid3=grid3, grad1=grad1, grad3=grad3, points=points, grid_voxel_coord=coord,
                grid_voxel_size=size, table=dict(mask=mask, keys=keys, g2v=g2v))
