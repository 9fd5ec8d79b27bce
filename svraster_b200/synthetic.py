"""Seeded synthetic sparse-voxel scenes and pinhole cameras.

The datasets the reference trains on are not available, so every workload here is
a procedurally generated octree that follows the reference's own data layout:

* ``octpath`` int64: 3 bits per level, level 1 in bits 45..47 (src/utils/octree_utils.py:13-22,
  cuda/src/utils.cu:129-158).
* voxel size ``scene_extent * 2**-level`` and centre ``scene_min + (ijk + 0.5) * size``
  (octree_utils.py:51-60, 99-126).
* grid points are the 8 corners of every voxel at level-16 integer resolution, merged by a
  lexicographic unique; ``vox_key[N, 8]`` indexes them with corner order ``x<<2 | y<<1 | z``
  (octree_utils.py:129-163, 203-222).

Cameras follow ``src/cameras.py``: OpenCV axes (x right, y down, z forward), ``c2w`` /
``w2c`` float32 4x4, ``tanfov = tan(fov / 2)``, principal point at the image centre.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MAX_NUM_LEVELS = 16


# ----------------------------------------------------------------------------- octree

def ijk_to_octpath(ijk: np.ndarray, level: np.ndarray) -> np.ndarray:
    """Octree path of voxels given integer coords at their own level (cuda/src/utils.cu:129-158)."""
    ijk = ijk.astype(np.int64)
    level = level.astype(np.int64).reshape(-1)
    path = np.zeros(len(level), dtype=np.int64)
    for l in range(MAX_NUM_LEVELS):
        bits = ((ijk[:, 0] >> l) & 1) << 2 | ((ijk[:, 1] >> l) & 1) << 1 | ((ijk[:, 2] >> l) & 1)
        path |= bits << (3 * l)
    return path << (3 * (MAX_NUM_LEVELS - level))


def octpath_to_ijk(path: np.ndarray, level: np.ndarray) -> np.ndarray:
    """Inverse of :func:`ijk_to_octpath` (cuda/src/utils.cu:160-189)."""
    level = level.astype(np.int64).reshape(-1)
    p = path.astype(np.int64).reshape(-1) >> (3 * (MAX_NUM_LEVELS - level))
    ijk = np.zeros((len(p), 3), dtype=np.int64)
    for l in range(MAX_NUM_LEVELS):
        b = p & 7
        ijk[:, 0] |= ((b >> 2) & 1) << l
        ijk[:, 1] |= ((b >> 1) & 1) << l
        ijk[:, 2] |= (b & 1) << l
        p = p >> 3
    return ijk


def build_grid_pts_link(ijk: np.ndarray, level: np.ndarray):
    """Corner grid points shared between voxels (octree_utils.py:129-163, 203-222).

    Returns ``(grid_pts_key int64[M,3], vox_key int64[N,8])`` with rows of
    ``grid_pts_key`` in lexicographic (x, y, z) order, as ``unique(dim=0)`` gives.
    """
    shift = (MAX_NUM_LEVELS - level.astype(np.int64)).reshape(-1, 1, 1)
    base = ijk.astype(np.int64).reshape(-1, 1, 3) << shift
    octant = np.array([[(k >> 2) & 1, (k >> 1) & 1, k & 1] for k in range(8)], dtype=np.int64)
    corners = base + (octant.reshape(1, 8, 3) << shift)          # [N, 8, 3], each < 2**16 + 1
    flat = (corners[..., 0] << 34) | (corners[..., 1] << 17) | corners[..., 2]
    uniq, inv = np.unique(flat.reshape(-1), return_inverse=True)
    key = np.stack([uniq >> 34, (uniq >> 17) & ((1 << 17) - 1), uniq & ((1 << 17) - 1)], axis=1)
    return key.astype(np.int64), inv.reshape(-1, 8).astype(np.int64)


# ----------------------------------------------------------------------------- SDFs

def sdf_sphere(p, r=0.5, c=(0.0, 0.0, 0.0)):
    return np.linalg.norm(p - np.asarray(c, dtype=np.float64), axis=-1) - r


def sdf_torus(p, R=0.35, r=0.12, c=(0.0, 0.0, 0.0)):
    q = p - np.asarray(c, dtype=np.float64)
    xz = np.sqrt(q[..., 0] ** 2 + q[..., 2] ** 2) - R
    return np.sqrt(xz ** 2 + q[..., 1] ** 2) - r


def sdf_spheres_torus(p):
    """Union of 3 spheres and a torus with radii in [0.2, 0.5] (mid-size workload)."""
    d = np.minimum(sdf_sphere(p, 0.5, (-0.3, 0.0, 0.0)), sdf_sphere(p, 0.3, (0.45, 0.3, 0.1)))
    d = np.minimum(d, sdf_sphere(p, 0.2, (0.2, -0.5, 0.4)))
    return np.minimum(d, sdf_torus(p, 0.45, 0.2, (0.1, 0.2, -0.35)))


def make_bumpy_sphere(n_bumps=64, amp=0.05, r=0.5, width=0.25, seed=0):
    rng = np.random.default_rng(seed)
    dirs = rng.normal(size=(n_bumps, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)

    def f(p):
        # |u - d|^2 = 2 - 2 u.d for unit u, d: one matrix product per chunk of points
        shape = p.shape[:-1]
        p = p.reshape(-1, 3)
        out = np.empty(len(p))
        for s in range(0, len(p), 1 << 20):
            q = p[s:s + (1 << 20)]
            n = np.linalg.norm(q, axis=-1)
            u = q / np.maximum(n, 1e-9)[:, None]
            h = amp * np.exp((2.0 * (u @ dirs.T) - 2.0) / width ** 2).sum(axis=1)
            out[s:s + len(q)] = n - (r + h)
        return out.reshape(shape)
    return f


# ----------------------------------------------------------------------------- scene

@dataclass
class Scene:
    octpath: np.ndarray          # int64 [N]
    octlevel: np.ndarray         # int8  [N]
    vox_center: np.ndarray       # f32   [N, 3]
    vox_size: np.ndarray         # f32   [N, 1]
    is_leaf: np.ndarray          # u8    [N]
    vox_key: np.ndarray          # int64 [N, 8]
    grid_pts_key: np.ndarray     # int64 [M, 3]
    grid_pts_xyz: np.ndarray     # f32   [M, 3]
    geo_grid_pts: np.ndarray     # f32   [M, 1]
    sh0: np.ndarray              # f32   [N, 3]
    shs: np.ndarray              # f32   [N, 15, 3]
    log_s: float
    scene_center: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    scene_extent: float = 2.0

    @property
    def n_vox(self):
        return len(self.octpath)

    @property
    def s_val(self):
        return float(np.exp(np.float32(self.log_s) * np.float32(10.0)))


def build_scene(sdf, lv_min, lv_max, seed=0, scene_extent=2.0, band=2.0, keep=None,
                kept_parent_frac=0.0, sh_degree=3, lv_max_fn=None, region=None):
    """Recursively subdivide cells with ``|sdf(centre)| < band * size`` from ``lv_min`` to ``lv_max``.

    Cells that are not subdivided stay as leaves when ``|sdf(centre)| < keep * size``
    (``keep=None`` keeps all of them); the rest count as pruned empty space, the state a
    trained scene reaches after the reference's max-weight pruning.

    ``kept_parent_frac`` re-inserts that fraction of the parents of finest-level leaves as
    non-leaf voxels, like the reference keeps deep parents on subdivision
    (src/sparse_voxel_gears/adaptive.py:59-63); those are culled by the preprocess.

    ``lv_max_fn(centres) -> int levels`` gives a finest level per region (clipped to
    [lv_min, lv_max]): a cell stops subdividing at its region's level.  ``region`` (lo, hi)
    keeps only the cells whose cube meets that box (a block of the same octree).
    """
    rng = np.random.default_rng(seed)
    smin = -0.5 * scene_extent
    n0 = 1 << lv_min
    g = np.stack(np.meshgrid(np.arange(n0), np.arange(n0), np.arange(n0), indexing="ij"), -1).reshape(-1, 3)
    cur_ijk, cur_lv = g.astype(np.int64), lv_min
    leaf_ijk, leaf_lv, parents = [], [], []
    while True:
        size = scene_extent * 2.0 ** -cur_lv
        if region is not None:
            c = smin + (cur_ijk + 0.5) * size
            meet = np.all((c + 0.5 * size >= np.asarray(region[0])) & (c - 0.5 * size <= np.asarray(region[1])), axis=1)
            cur_ijk = cur_ijk[meet]
        c = smin + (cur_ijk + 0.5) * size
        d = np.abs(sdf(c))
        if cur_lv == lv_max:
            kept = cur_ijk if keep is None else cur_ijk[d < keep * size]
            leaf_ijk.append(kept); leaf_lv.append(np.full(len(kept), cur_lv))
            break
        near = d < band * size
        if lv_max_fn is not None:
            near &= np.clip(lv_max_fn(c), lv_min, lv_max) > cur_lv
        stay = ~near if keep is None else (~near) & (d < keep * size)
        leaf_ijk.append(cur_ijk[stay]); leaf_lv.append(np.full(int(stay.sum()), cur_lv))
        sub = cur_ijk[near]
        if cur_lv + 1 == lv_max and kept_parent_frac > 0 and len(sub):
            pick = rng.random(len(sub)) < kept_parent_frac
            parents.append(sub[pick])
        octant = np.array([[(k >> 2) & 1, (k >> 1) & 1, k & 1] for k in range(8)], dtype=np.int64)
        cur_ijk = ((sub[:, None, :] << 1) + octant[None]).reshape(-1, 3)
        cur_lv += 1
    ijk = np.concatenate(leaf_ijk)
    lv = np.concatenate(leaf_lv).astype(np.int64)
    leaf = np.ones(len(ijk), np.uint8)
    if parents:
        pij = np.concatenate(parents)
        ijk = np.concatenate([ijk, pij]); lv = np.concatenate([lv, np.full(len(pij), lv_max - 1)])
        leaf = np.concatenate([leaf, np.zeros(len(pij), np.uint8)])
    # shuffle so voxel ids are not spatially ordered (as after many prune/subdivide rounds)
    perm = rng.permutation(len(ijk))
    ijk, lv, leaf = ijk[perm], lv[perm], leaf[perm]

    size = (scene_extent * np.exp2(-lv.astype(np.float64))).astype(np.float32)
    center = (smin + (ijk + 0.5) * size[:, None].astype(np.float64)).astype(np.float32)
    octpath = ijk_to_octpath(ijk, lv)
    gkey, vkey = build_grid_pts_link(ijk, lv)
    finest = scene_extent * 2.0 ** -MAX_NUM_LEVELS
    gxyz = (smin + gkey * finest).astype(np.float32)
    h_min = scene_extent * 2.0 ** -lv_max
    geo = sdf(gxyz.astype(np.float64)) + rng.normal(0.0, 0.01 * h_min, size=len(gxyz))
    N = len(ijk)
    sh0 = rng.uniform(-1.0, 1.0, size=(N, 3)).astype(np.float32)
    n_rest = (sh_degree + 1) ** 2 - 1
    shs = rng.normal(0.0, 0.05, size=(N, n_rest, 3)).astype(np.float32)
    log_s = 0.1 * math.log(math.log(99.0) / h_min / 4.0)
    return Scene(octpath=octpath, octlevel=lv.astype(np.int8), vox_center=center,
                 vox_size=size.reshape(-1, 1), is_leaf=leaf, vox_key=vkey, grid_pts_key=gkey,
                 grid_pts_xyz=gxyz, geo_grid_pts=geo.astype(np.float32).reshape(-1, 1),
                 sh0=sh0, shs=shs, log_s=log_s, scene_extent=scene_extent)


# ----------------------------------------------------------------------------- cameras

@dataclass
class Camera:
    width: int
    height: int
    fovx: float
    fovy: float
    c2w: np.ndarray      # f32 [4, 4]
    w2c: np.ndarray      # f32 [4, 4]
    near: float = 0.02

    @property
    def tanfovx(self):
        return math.tan(self.fovx * 0.5)

    @property
    def tanfovy(self):
        return math.tan(self.fovy * 0.5)

    @property
    def cx(self):
        return self.width * 0.5

    @property
    def cy(self):
        return self.height * 0.5

    @property
    def position(self):
        return self.c2w[:3, 3]

    @property
    def lookat(self):
        return self.c2w[:3, 2]


def look_at_camera(pos, width, height, fovx_deg=50.0, target=(0.0, 0.0, 0.0)):
    pos = np.asarray(pos, np.float64)
    f = np.asarray(target, np.float64) - pos
    f /= np.linalg.norm(f)
    up = np.array([0.0, 0.0, 1.0])
    if abs(f @ up) > 0.99:
        up = np.array([0.0, 1.0, 0.0])
    right = np.cross(f, up); right /= np.linalg.norm(right)
    down = np.cross(f, right)
    c2w = np.eye(4)
    c2w[:3, 0], c2w[:3, 1], c2w[:3, 2], c2w[:3, 3] = right, down, f, pos
    w2c = np.linalg.inv(c2w)
    fovx = math.radians(fovx_deg)
    fovy = 2 * math.atan(math.tan(fovx / 2) * height / width)
    # the reference inverts w2c in float32 on the device (src/cameras.py:146-149)
    w2c32 = w2c.astype(np.float32)
    c2w32 = np.linalg.inv(w2c32.astype(np.float64)).astype(np.float32)
    return Camera(width, height, fovx, fovy, c2w32, w2c32)


def ring_cameras(n, radius, width, height, fovx_deg=50.0, elev_deg=20.0, phase=0.0):
    cams = []
    for i in range(n):
        az = phase + 2 * math.pi * i / n
        el = math.radians(elev_deg)
        p = radius * np.array([math.cos(az) * math.cos(el), math.sin(az) * math.cos(el), math.sin(el)])
        cams.append(look_at_camera(p, width, height, fovx_deg))
    return cams


def fibonacci_points(n, radius):
    ga = math.pi * (3.0 - math.sqrt(5.0))
    pts = []
    for i in range(n):
        z = 1 - 2 * (i + 0.5) / n
        r = math.sqrt(max(0.0, 1 - z * z))
        pts.append(radius * np.array([math.cos(ga * i) * r, math.sin(ga * i) * r, z]))
    return pts


def fibonacci_cameras(n, radius, width, height, fovx_deg=50.0):
    return [look_at_camera(p, width, height, fovx_deg) for p in fibonacci_points(n, radius)]


# ----------------------------------------------------------------------------- workloads

def scene_small(seed=0):
    """Unit-sphere (r=0.5) scene at levels 5-7."""
    return build_scene(lambda p: sdf_sphere(p, 0.5), 5, 7, seed=seed, band=1.0, keep=2.0,
                       kept_parent_frac=0.05)


def scene_mid(seed=0):
    """3 spheres + torus at levels 6-10 (about a million voxels)."""
    return build_scene(sdf_spheres_torus, 6, 10, seed=seed, band=0.35, keep=2.0, kept_parent_frac=0.02)


def scene_precision(seed=0):
    """The mid-size procedure (3 spheres + torus) carried to level 11: about 7.9M voxels."""
    return build_scene(sdf_spheres_torus, 6, 11, seed=seed, band=0.42, keep=1.6, kept_parent_frac=0.02)


def scene_batched(seed=0):
    """Sphere with 64 Gaussian bumps (amplitude 0.05) at levels 7-11, about 4M voxels."""
    return build_scene(make_bumpy_sphere(seed=seed), 7, 11, seed=seed, band=0.42, keep=1.1, kept_parent_frac=0.02)


ROOM_HALF = (2.0, 1.5, 1.25)          # 4 x 3 x 2.5 room


def sdf_box(p, c, half):
    q = np.abs(p - np.asarray(c, dtype=np.float64)) - np.asarray(half, dtype=np.float64)
    outside = np.linalg.norm(np.maximum(q, 0.0), axis=-1)
    return outside + np.minimum(q.max(axis=-1), 0.0)


def make_room(n_objects=20, n_fine=4, seed=0):
    """An indoor-like SDF: the inside of an axis-aligned 4 x 3 x 2.5 box room (walls solid)
    with ``n_objects`` seeded boxes and spheres standing inside it.  Returns (sdf, objects_sdf,
    fine_sdf): the scene, the union of the objects, and the union of the first ``n_fine``
    objects (the ones refined to the finest level)."""
    rng = np.random.default_rng(seed)
    hx, hy, hz = ROOM_HALF
    objs = []
    for k in range(n_objects):
        r = rng.uniform(0.12, 0.35)
        c = rng.uniform([-hx + 0.5, -hy + 0.5, -hz + r], [hx - 0.5, hy - 0.5, hz - 0.5])
        if k % 2 == 0:
            objs.append(("sphere", c, r))
        else:
            objs.append(("box", c, rng.uniform(0.1, 0.35, size=3)))

    def one(p, o):
        kind, c, sz = o
        return sdf_sphere(p, sz, c) if kind == "sphere" else sdf_box(p, c, sz)

    cache = {}

    def union(p, sel):
        # the octree builder asks for the scene and the objects at the same centres in a row
        key = (id(p), p.shape, len(sel))
        if cache.get("key") == key:
            return cache["val"]
        q = np.asarray(p, dtype=np.float64)
        d = np.full(q.shape[:-1], np.inf)
        for o in sel:
            d = np.minimum(d, one(q, o))
        cache["key"], cache["val"] = key, d
        return d

    def room(p):
        q = np.asarray(p, dtype=np.float64)
        walls = np.minimum(np.minimum(hx - np.abs(q[..., 0]), hy - np.abs(q[..., 1])), hz - np.abs(q[..., 2]))
        return np.minimum(walls, union(p, objs))

    return room, (lambda p: union(p, objs)), (lambda p: union(p, objs[:n_fine]))


def scene_full(seed=0):
    """Full reconstruction workload: the 4 x 3 x 2.5 room with 20 boxes and spheres in the
    scene cube [-2, 2]^3 (inside extent 4), levels 8-12: walls refined to level 10, objects to
    level 11, four of them to level 12; empty space pruned; about 12M voxels."""
    room, objs, fine = make_room(seed=seed)

    def lv_max(c):
        lv = np.full(len(c), 10)
        lv[np.abs(objs(c)) < 0.03] = 11
        lv[np.abs(fine(c)) < 0.02] = 12
        return lv
    return build_scene(room, 8, 12, seed=seed, scene_extent=4.0, band=0.46, keep=1.1, kept_parent_frac=0.02,
                       lv_max_fn=lv_max)


def full_block_region(seed=0, margin=0.08):
    """A box around the first of the objects refined to level 12 in scene_full."""
    rng = np.random.default_rng(seed)
    hx, hy, hz = ROOM_HALF
    r = rng.uniform(0.12, 0.35)
    c = rng.uniform([-hx + 0.5, -hy + 0.5, -hz + r], [hx - 0.5, hy - 0.5, hz - 0.5])
    lo = c - r - margin
    return (lo, lo + np.array([r + margin, 2 * (r + margin), 2 * (r + margin)]))


def scene_full_block(seed=0):
    """A block of the full reconstruction workload's octree (scene_full's procedure restricted
    to a box that cuts through one level-12 object and its surroundings), small enough for
    reference checks on the CPU."""
    room, objs, fine = make_room(seed=seed)

    def lv_max(c):
        lv = np.full(len(c), 10)
        lv[np.abs(objs(c)) < 0.03] = 11
        lv[np.abs(fine(c)) < 0.02] = 12
        return lv
    return build_scene(room, 8, 12, seed=seed, scene_extent=4.0, band=0.46, keep=1.1, kept_parent_frac=0.02,
                       lv_max_fn=lv_max, region=full_block_region(seed))


def room_cameras(n, width=1024, height=768, fovx_deg=70.0, seed=0):
    """n views from inside the room: positions on an ellipse at mid height (clear of the
    objects' extent in z only where they stand low), each looking at a seeded point on the far
    walls or floor."""
    rng = np.random.default_rng(seed)
    hx, hy, hz = ROOM_HALF
    cams = []
    for i in range(n):
        az = 2 * math.pi * i / n
        pos = np.array([0.55 * hx * math.cos(az), 0.55 * hy * math.sin(az), rng.uniform(0.3, 0.8) * hz])
        tgt = np.array([rng.uniform(-hx, hx), rng.uniform(-hy, hy), rng.uniform(-hz, 0.2 * hz)])
        tgt[0] = -np.sign(pos[0] + 1e-9) * abs(tgt[0])
        cams.append(look_at_camera(pos, width, height, fovx_deg, target=tuple(tgt)))
    return cams


MIXED_RESOLUTIONS = ((480, 360), (960, 540), (1280, 720), (1920, 1080))


def mixed_resolution_cameras(n=64, radius=3.0, fovx_deg=50.0, seed=0):
    """n views on a Fibonacci sphere, n/4 at each of MIXED_RESOLUTIONS, shuffled by `seed`."""
    sizes = [MIXED_RESOLUTIONS[i % len(MIXED_RESOLUTIONS)] for i in range(n)]
    order = np.random.default_rng(seed).permutation(n)
    return [look_at_camera(p, sizes[order[i]][0], sizes[order[i]][1], fovx_deg=fovx_deg)
            for i, p in enumerate(fibonacci_points(n, radius))]


def scene_tiny(seed=0, lv_min=3, lv_max=5):
    """A few thousand voxels; sized so the pure-C oracle finishes in well under a second."""
    return build_scene(lambda p: sdf_sphere(p, 0.5), lv_min, lv_max, seed=seed, band=1.0, keep=3.0,
                       kept_parent_frac=0.1)
