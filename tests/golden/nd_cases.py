"""Seeded inputs of the normal-from-depth consistency-loss cases (shared by the generator and
the tests): a camera looking at a sphere of radius 0.6, depth planes from the ray-sphere hit
(plus noise; misses at a far plane), rendered normals near the sphere normal with noise and
some flipped, transmittance small on the sphere and 1 off it."""
from __future__ import annotations

import numpy as np

from svraster_b200 import synthetic as S

# mode "dmean": NormalDepthConsistencyLoss (depth plane 0, alpha weighting, ks, tol_deg);
# mode "dmed": NormalMedianConsistencyLoss (depth plane 2, ks 3, no tolerance)
ND_CASES = {
    "dmean_ks3": dict(mode="dmean", W=64, H=48, ks=3, tol_deg=90.0, seed=0, phase=0.2),
    "dmean_ks5_tol60": dict(mode="dmean", W=45, H=37, ks=5, tol_deg=60.0, seed=1, phase=1.1),
    "dmed": dict(mode="dmed", W=53, H=40, ks=3, tol_deg=None, seed=2, phase=2.3),
}


def nd_camera(case):
    return S.ring_cameras(1, 2.2, case["W"], case["H"], fovx_deg=55.0, phase=case["phase"])[0]


def nd_inputs(case, c2w=None, cam=None):
    """(depth f32[4,H,W], normal f32[3,H,W], T f32[1,H,W]) for the case seen by ``cam`` (the
    case's camera by default); ray directions from ``c2w`` (the reference camera's float32
    inverse of w2c, when given)."""
    cam = nd_camera(case) if cam is None else cam
    W, H = case["W"], case["H"]
    c2w = (cam.c2w if c2w is None else c2w).astype(np.float64)
    rng = np.random.default_rng(case["seed"] + 40)
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    cam_d = np.stack([(x + 0.5 - cam.cx) * 2 * cam.tanfovx / W, (y + 0.5 - cam.cy) * 2 * cam.tanfovy / H,
                      np.ones_like(x)], 0)
    rd = np.einsum("ij,jhw->ihw", c2w[:3, :3], cam_d)
    o = c2w[:3, 3].reshape(3, 1, 1)
    a = (rd * rd).sum(0)
    b = 2 * (rd * o).sum(0)
    c = (o * o).sum() - 0.6 ** 2
    disc = b * b - 4 * a * c
    hit = disc > 0
    t = np.where(hit, (-b - np.sqrt(np.maximum(disc, 0))) / (2 * a), 3.0)
    depth = np.zeros((4, H, W))
    depth[0] = t + 1e-3 * rng.normal(size=(H, W))
    depth[1] = rng.normal(size=(H, W))
    depth[2] = t + 2e-3 * rng.normal(size=(H, W))
    depth[3] = rng.normal(size=(H, W))
    p = o + rd * t
    n = p / np.maximum(np.linalg.norm(p, axis=0, keepdims=True), 1e-9)
    n = n + 0.2 * rng.normal(size=n.shape)
    n[:, rng.random((H, W)) < 0.1] *= -1.0
    T = np.where(hit, 0.3 * rng.random((H, W)), 1.0)[None]
    return depth.astype(np.float32), n.astype(np.float32), T.astype(np.float32)
