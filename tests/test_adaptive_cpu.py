"""Pruning / subdivision goldens (the reference's own torch code on the CPU,
tests/golden/make_golden_adaptive.py) against this repository's NumPy grid-point link."""
from __future__ import annotations

import os

import numpy as np

from svraster_b200 import synthetic as S
from tests.golden.adaptive_cases import scene

GOLD = os.path.join(os.path.dirname(__file__), "golden", "adaptive.npz")


def test_numpy_grid_link_matches_reference_golden():
    g = np.load(GOLD)
    sc = scene()
    assert int(g["digest"]) == sc.n_vox
    ijk = S.octpath_to_ijk(sc.octpath, sc.octlevel.astype(np.int64))
    key, vkey = S.build_grid_pts_link(ijk, sc.octlevel)
    assert np.array_equal(key, g["link_key"])
    assert np.array_equal(vkey, g["link_vox_key"])
    # the scene's own link is the same one
    assert np.array_equal(sc.vox_key, g["link_vox_key"])


def test_golden_subdivision_shapes():
    g = np.load(GOLD)
    n0 = int(g["digest"])
    n1 = len(g["sub_octpath"])
    assert n1 > n0 and len(g["prune_octpath"]) < n1
    assert g["sub_vox_key"].shape == (n1, 8)
    assert g["sub__geo_grid_pts"].shape[0] == len(g["sub_grid_pts_key"])
