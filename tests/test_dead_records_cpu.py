"""The render kernels give no candidate pixels to a record whose SDF corners put every pair
of it below MIN_ALPHA (record_dead in svraster_b200/csrc/render_pairs.cuh).  The forward and
the adjoint skip such pairs anyway (forward.cu:304, backward.cu:428), so the outputs stay the
same bit for bit -- provided the rule never drops a pair whose alpha reaches MIN_ALPHA.  This
checks that on the CPU: float32 restatements of the rule and of a pair's alpha (slab test,
entry point and three sub-steps as the forward takes them, entry and exit as the adjoint
does) on seeded voxels placed at the rule's thresholds, with rays through their faces, edges
and corners and at grazing angles."""
import numpy as np
import pytest

f32 = np.float32
MIN_ALPHA = f32(1e-5)


def record_dead(g, s):
    lo, hi = g.min(-1), g.max(-1)
    margin = f32(0.05) * (hi - lo) + f32(1e-4) * np.maximum(np.abs(lo), np.abs(hi))
    return (s > 0) & ((s * (lo - margin) >= f32(16)) | (s * (hi + margin) <= f32(-30)))


def tri(q):
    x, y, z = q[..., 0], q[..., 1], q[..., 2]
    wx = (f32(1) - x, x); wy = (f32(1) - y, y); wz = (f32(1) - z, z)
    return np.stack([wx[i >> 2] * wy[(i >> 1) & 1] * wz[i & 1] for i in range(8)], -1)


def interp(g, w):
    acc = np.zeros(w.shape[:-1], f32)
    for i in range(8):
        acc = (acc + g[..., i] * w[..., i]).astype(f32)
    return acc


def phi(s, sdf):
    with np.errstate(over="ignore"):
        return (f32(1) / (f32(1) + np.exp(-s * sdf))).astype(f32)


def pair_alphas(c, l, g, s, ro, rd):
    """(forward alpha, adjoint alpha, candidate) of rays ro + t rd through voxels (c, l)."""
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        rd_inv = (f32(1) / rd).astype(f32)
        r = (f32(0.5) * l)[..., None]
        d = (c - ro).astype(f32)
        t0, t1 = ((d - r) * rd_inv).astype(f32), ((d + r) * rd_inv).astype(f32)
        a = np.fmax(np.fmax(np.fmin(t0, t1)[..., 0], np.fmin(t0, t1)[..., 1]), np.fmin(t0, t1)[..., 2])
        b = np.fmin(np.fmin(np.fmax(t0, t1)[..., 0], np.fmax(t0, t1)[..., 1]), np.fmax(t0, t1)[..., 2])
        cand = ~(a > b)
        linv = (f32(1) / l)[..., None]
        lo3 = (c - f32(0.5) * l[..., None]).astype(f32)
        qe = (((ro + a[..., None] * rd) - lo3) * linv).astype(f32)
        step = ((((b - a)[..., None] * rd) / f32(3)) * linv).astype(f32)
        ph_e = phi(s, interp(g, tri(qe)))
        ph = ph_e
        for k in range(1, 4):
            ph = phi(s, interp(g, tri((qe + step * f32(k)).astype(f32))))
        fwd = np.fmax((ph_e - ph) / (ph_e + f32(1e-6)), f32(0))
        qx = (((ro + b[..., None] * rd) - lo3) * linv).astype(f32)
        ph_x = phi(s, interp(g, tri(qx)))
        bwd = np.fmax((ph_e - ph_x) / (ph_e + f32(1e-6)), f32(0))
    return fwd, bwd, cand


@pytest.mark.parametrize("side", ["outside", "inside"])
def test_dead_records_have_no_pair_at_min_alpha(side):
    rng = np.random.default_rng(1 if side == "outside" else 2)
    n = 200_000
    l = (f32(2) ** -rng.integers(4, 15, size=n)).astype(f32)          # levels 4-14 of a 2-unit scene
    c = rng.uniform(-1, 1, size=(n, 3)).astype(f32)
    s = (f32(10) ** rng.uniform(1, 4, size=n)).astype(f32)             # 10 .. 1e4
    spread = (rng.uniform(0, 3, size=(n, 1)) * l[:, None]).astype(f32)  # corner spread ~ voxel size
    thr = f32(16) if side == "outside" else f32(-30)
    # centre the corners so that the rule's bound lands just on either side of the threshold
    base = (thr / s * rng.uniform(0.3, 1.2, size=n)).astype(f32)
    g = (base[:, None] + (rng.uniform(0, 1, size=(n, 8)) - (0 if side == "outside" else 1)) * spread).astype(f32)
    dead = record_dead(g, s)
    assert dead.sum() > n // 10 and (~dead).sum() > n // 10
    # rays from a camera at distance 3 through random points of the voxel, some along its
    # faces and edges (points on the boundary), some grazing
    cam = rng.normal(size=(n, 3)).astype(f32)
    cam = (cam / np.linalg.norm(cam, axis=1, keepdims=True) * f32(3)).astype(f32)
    u = rng.uniform(-0.5, 0.5, size=(n, 3)).astype(f32)
    snap = rng.random(size=(n, 3)) < 0.3
    u = np.where(snap, np.sign(u) * f32(0.5), u).astype(f32)
    target = (c + u * l[:, None]).astype(f32)
    rd = (target - cam).astype(f32)
    graze = rng.random(n) < 0.2
    rd[graze, rng.integers(0, 3, size=graze.sum())] = f32(0)
    fwd, bwd, cand = pair_alphas(c, l, g, s, cam, rd)
    sel = dead & cand
    assert sel.sum() > 1000
    assert np.all(fwd[sel] < MIN_ALPHA) and np.all(bwd[sel] < MIN_ALPHA)
    # the cases are not vacuous: live records below the threshold reach MIN_ALPHA on some rays
    assert np.any((fwd >= MIN_ALPHA) & cand & ~dead)
