"""Seeded inputs of the checkpoint-format golden cases (shared by the generator and tests)."""
from __future__ import annotations

import numpy as np

from svraster_b200 import synthetic as S

# value sets for the 8-bit codebook: a plain normal set, heavy ties, fewer values than codebook
# entries, a multi-dimensional SH-like block, the small scene's SDF grid, a skewed set, one value
QUANT_CASES = ("normal", "ties", "small", "shblock", "geo", "skewed", "one")


def quant_values(name):
    rng = np.random.default_rng(QUANT_CASES.index(name) + 21)
    if name == "normal":
        return rng.normal(size=20000).astype(np.float32)
    if name == "ties":
        return (np.round(rng.laplace(size=30011) * 8.0) / 8.0).astype(np.float32)
    if name == "small":
        return rng.normal(size=100).astype(np.float32)
    if name == "shblock":
        return (0.3 * rng.normal(size=(700, 1, 3))).astype(np.float32)
    if name == "geo":
        return model_fields()["_geo_grid_pts"].copy()
    if name == "skewed":
        return rng.exponential(size=9000).astype(np.float32) ** 3
    if name == "one":
        return np.array([0.25], np.float32)
    raise KeyError(name)


def small_scene():
    return S.scene_tiny(seed=3, lv_min=2, lv_max=4)


def model_fields():
    """The attributes SVInOut.save reads (io.py:23-36), for the seeded small scene."""
    sc = small_scene()
    N = sc.n_vox
    return dict(active_sh_degree=3, ss=1.5,
                scene_center=np.zeros(3, np.float32),
                inside_extent=np.array(sc.scene_extent, np.float32),
                scene_extent=np.array(sc.scene_extent, np.float32),
                octpath=sc.octpath.reshape(N, 1).astype(np.int64),
                octlevel=sc.octlevel.reshape(N, 1).astype(np.int8),
                _geo_grid_pts=sc.geo_grid_pts.reshape(-1, 1).astype(np.float32),
                _sh0=sc.sh0.astype(np.float32), _shs=sc.shs.astype(np.float32),
                _log_s=np.array(sc.log_s, np.float32),
                is_leaf=sc.is_leaf.reshape(N, 1).astype(bool))
