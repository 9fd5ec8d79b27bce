"""Seeded inputs of the pruning / subdivision golden case (shared by the generator and tests)."""
from __future__ import annotations

import numpy as np

from svraster_b200 import synthetic as S

SUBDIV_FRAC = 0.08
PRUNE_FRAC = 0.05
# levels 3-5 with outside level -4: level-5 voxels sit at relative depth 9, so subdividing
# them keeps the parent as a non-leaf voxel (adaptive.py:59-63)
OUTSIDE_LEVEL = -4


def scene():
    return S.scene_tiny(seed=2)


def model_inputs(sc):
    rng = np.random.default_rng(4)
    N = sc.n_vox
    return dict(octpath=sc.octpath.reshape(-1, 1).astype(np.int64),
                octlevel=sc.octlevel.reshape(-1, 1).astype(np.int8),
                vox_center=sc.vox_center.astype(np.float32),
                vox_size=sc.vox_size.reshape(-1, 1).astype(np.float32),
                subdiv_meta=rng.random((N, 1)).astype(np.float32),
                is_leaf=sc.is_leaf.reshape(-1, 1).astype(bool),
                _sh0=sc.sh0.astype(np.float32), _shs=sc.shs[:, :3].astype(np.float32),
                _subdiv_p=rng.random((N, 1)).astype(np.float32),
                _geo_grid_pts=sc.geo_grid_pts.reshape(-1, 1).astype(np.float32))
