"""Seeded inputs of the TSDF / marching-cubes golden cases (generator and tests share them)."""
from __future__ import annotations

import hashlib

import numpy as np

from svraster_b200 import synthetic as S

TSDF_CASES = {
    "tsdf_a": dict(seed=0, n_views=4, W=64, H=48, trunc_vox=5.0, per_point=False, use_trunc=True,
                   crop_border=0.01, alpha_thres=0.5, depth_weight=False, border_weight=False),
    "tsdf_b": dict(seed=1, n_views=3, W=80, H=60, trunc_vox=3.0, per_point=True, use_trunc=False,
                   crop_border=0.05, alpha_thres=0.3, depth_weight=True, border_weight=True),
}
MC_CASES = {
    "mc_a": dict(kind="tiny", seed=0, iso=0.0, subset=1, specials=False),
    "mc_b": dict(kind="small", seed=1, iso=0.01, subset=2, specials=True),
    # the full reconstruction workload's procedure on a block: the level-12 voxels only
    "mc_full_block": dict(kind="full_block", seed=0, iso=0.0, subset=1, specials=False, level=12, compact=True),
}


def mesh_digest(verts, faces, n_sample=2048, seed=0):
    """Compact golden of a large mesh: SHA-256 of the exact bytes of the vertices (float32
    [V,3]) and faces (int64 [F,3]), the counts, and a seeded sample of rows for diagnostics."""
    verts = np.ascontiguousarray(verts, dtype=np.float32)
    faces = np.ascontiguousarray(faces, dtype=np.int64)
    rng = np.random.default_rng(seed)
    vi = np.sort(rng.choice(len(verts), min(n_sample, len(verts)), replace=False))
    fi = np.sort(rng.choice(len(faces), min(n_sample, len(faces)), replace=False))
    return dict(verts_sha256=hashlib.sha256(verts.tobytes()).hexdigest(),
                faces_sha256=hashlib.sha256(faces.tobytes()).hexdigest(),
                n_verts=len(verts), n_faces=len(faces), vert_rows=vi, verts_sample=verts[vi], face_rows=fi,
                faces_sample=faces[fi])


def _digest(arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def tsdf_inputs(case):
    from oracle import oracle as O
    sc = S.scene_tiny(seed=case["seed"])
    cams = S.ring_cameras(case["n_views"], 3.0, case["W"], case["H"], phase=0.7 + case["seed"])
    depths, alphas = [], []
    for cam in cams:
        nd, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
        keys, vals, ranges = O.binning(cam, sc.octpath, nd, bb, bits)
        geos = O.gather_geo(np.arange(sc.n_vox), sc.vox_key, sc.geo_grid_pts, sc.n_vox)
        rgbs = O.sh_eval(3, None, sc.vox_center, cam.position, sc.sh0, sc.shs)
        f = O.render_fwd(cam, np.zeros(3, np.float32), 3, True, True, ranges, vals, bb, sc.vox_center,
                         sc.vox_size, geos, rgbs, sc.s_val)
        depths.append(f["depth"][[2]].astype(np.float32))              # median depth
        alphas.append((np.float32(1.0) - f["T"]).astype(np.float32))   # alpha = 1 - T
    finest = sc.scene_extent * 2.0 ** -int(sc.octlevel.max())
    trunc = case["trunc_vox"] * finest
    xyz = sc.grid_pts_xyz.astype(np.float32)
    if case["per_point"]:
        rng = np.random.default_rng(case["seed"] + 3)
        bandwidth = (trunc * rng.uniform(0.5, 1.5, size=len(xyz))).astype(np.float32)
    else:
        bandwidth = float(trunc)
    arrays = [xyz] + depths + alphas + [c.w2c for c in cams] + ([bandwidth] if case["per_point"] else [])
    return dict(scene=sc, cams=cams, depths=depths, alphas=alphas, xyz=xyz, bandwidth=bandwidth,
                digest=_digest(arrays))


def mc_inputs(case):
    if case["kind"] == "full_block":
        sc = S.scene_full_block(seed=case["seed"])
    else:
        sc = S.scene_tiny(seed=case["seed"]) if case["kind"] == "tiny" else S.scene_small(seed=case["seed"])
    val = sc.geo_grid_pts.reshape(-1).astype(np.float32).copy()
    if case["specials"]:
        rng = np.random.default_rng(case["seed"] + 9)
        k = len(val)
        val[rng.choice(k, k // 200, replace=False)] = np.float32(case["iso"])        # exact iso hits
        val[rng.choice(k, k // 500, replace=False)] = np.nan                          # NaN corners
    vox_key = sc.vox_key
    if "level" in case:
        vox_key = vox_key[sc.octlevel.reshape(-1) == case["level"]]
    vox_key = vox_key[:: case["subset"]].astype(np.int64).copy()
    xyz = sc.grid_pts_xyz.astype(np.float32)
    return dict(val=val, xyz=xyz, vox_key=vox_key, digest=_digest([val, xyz, vox_key]))
