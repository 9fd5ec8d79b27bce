"""Binning with dense (voxel, octant) ranks (``svr_bin_and_sort_ranked``, ``raster.RankTable``)
gives the record order, tile ranges and images of the plain trimmed-rank key bit for bit."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from svraster_b200 import synthetic as S
from svraster_b200.raster import RankTable, RasterState, rank_shift
from svraster_b200.step import BatchedTrainStep

pytestmark = pytest.mark.gpu


def _bin_both(sc, cams, capacity=None):
    step = BatchedTrainStep(sc, cams, device="cuda", dense_ranks=False)
    out = []
    for table in (None, RankTable(step.octpath, step.path_or_all)):
        st = RasterState(step.views, step.N, step.dev)
        st.preprocess(step.octpath, step.centers, step.lengths, step.is_leaf)
        if capacity is None:
            st.bin(step.octpath, rank_table=table)
        else:
            st.bin(step.octpath, capacity=capacity, path_or=step.path_or_all, rank_table=table)
        vals, ranges, _, _ = st.binning_fields()
        color, _, _, T, _ = st.render(3, True, True, step.centers, step.lengths,
                                      step.grid.reshape(-1)[step.vox_key].contiguous(),
                                      torch.rand(step.V * step.N, 3, device="cuda", generator=torch.Generator(
                                          device="cuda").manual_seed(0)), step.s_val, rgb_per_view=True)
        out.append((vals.cpu().numpy(), ranges.cpu().numpy(), color.cpu().numpy(), T.cpu().numpy(),
                    table.bits if table is not None else None))
    return out


@pytest.mark.parametrize("seed,n_views,W,H", [(1, 3, 200, 150), (5, 1, 333, 257)])
def test_dense_rank_binning_is_bit_identical(seed, n_views, W, H):
    sc = S.scene_small(seed=seed)
    cams = S.ring_cameras(n_views, 3.0, W, H, fovx_deg=50.0, phase=0.2 * seed)
    (v0, r0, c0, t0, _), (v1, r1, c1, t1, bits) = _bin_both(sc, cams)
    assert bits <= 24 and len(v0) > 1000
    assert np.array_equal(v0, v1) and np.array_equal(r0, r1)
    assert np.array_equal(c0, c1) and np.array_equal(t0, t1)


def test_dense_rank_binning_with_capacity():
    sc = S.scene_small(seed=2)
    cams = S.ring_cameras(2, 3.0, 160, 120, fovx_deg=50.0)
    (v0, r0, _, _, _), (v1, r1, _, _, _) = _bin_both(sc, cams, capacity=2_000_000)
    assert np.array_equal(v0, v1) and np.array_equal(r0, r1)


def test_rank_table_is_order_preserving():
    """table[v*8+q] orders and ties exactly as (path ^ octant pattern) >> shift."""
    sc = S.scene_small(seed=3)
    paths = torch.as_tensor(sc.octpath.reshape(-1), device="cuda")
    path_or = int(np.bitwise_or.reduce(sc.octpath.reshape(-1).astype(np.int64).view(np.uint64)))
    tab = RankTable(paths, path_or)
    shift = rank_shift(path_or)
    rep = [sum(q << (3 * l) for l in range(16)) for q in range(8)]
    p = sc.octpath.reshape(-1).astype(np.uint64)
    rank = np.stack([(p ^ np.uint64(rep[q])) >> np.uint64(shift) for q in range(8)], 1).reshape(-1)
    _, inv = np.unique(rank, return_inverse=True)
    assert np.array_equal(tab.table.cpu().numpy().astype(np.int64), inv.reshape(-1))
    assert (1 << tab.bits) >= inv.max() + 1
