"""Binning by per-tile sort (``svr_bin_tiles``, ``raster.PairOrder``): the pair-order table
equals the reference order of (voxel, octant) pairs, and the record order, tile ranges and
images equal those of the global radix sort (``svr_bin_and_sort``) and of the oracle bit for
bit, for tiles sorted in shared memory and tiles above its capacity, with and without a
record capacity, on small scenes and on all 8 views of the mid-size workload."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from svraster_b200 import synthetic as S
from svraster_b200.raster import PairOrder, RasterState
from tests.helpers import oracle_view, oracle_inputs, torch_scene, cam_dict

pytestmark = pytest.mark.gpu


def _reference_pair_order(octpath):
    """Position of pair s = 8 v + q when sorted by (path ^ repeat3(q), s)."""
    p = octpath.reshape(-1).astype(np.int64).view(np.uint64)
    rep = [np.uint64(sum(q << (3 * l) for l in range(16))) for q in range(8)]
    rank = np.stack([p ^ rep[q] for q in range(8)], 1).reshape(-1)
    s = np.arange(rank.size, dtype=np.int64)
    order = np.lexsort((s, rank))
    pos = np.empty_like(order)
    pos[order] = np.arange(order.size)
    return pos


def _bin(sc, cams, pair_order, capacity=None):
    ts = torch_scene(sc)
    views = [cam_dict(c) for c in cams]
    st = RasterState(views, sc.n_vox, torch.device("cuda"))
    st.preprocess(ts["octpath"], ts["centers"], ts["lengths"], ts["is_leaf"])
    if capacity is None:
        st.bin(ts["octpath"], pair_order=pair_order)
    else:
        por = int(np.bitwise_or.reduce(sc.octpath.reshape(-1).astype(np.int64).view(np.uint64)))
        st.bin(ts["octpath"], capacity=capacity, path_or=por, pair_order=pair_order)
    vals, ranges, _, _ = st.binning_fields()
    torch.cuda.synchronize()
    return st, vals.cpu().numpy().view(np.uint32), ranges.cpu().numpy().view(np.uint32)


def test_pair_order_table_matches_reference_order():
    sc = S.scene_small(seed=3)
    po = PairOrder(torch.as_tensor(sc.octpath.reshape(-1), device="cuda"))
    got = po.pos.cpu().numpy().astype(np.int64)
    ref = _reference_pair_order(sc.octpath).reshape(sc.n_vox, 8).T.reshape(-1)   # octant-major
    assert np.array_equal(got, ref)
    assert (1 << po.bits) >= 8 * sc.n_vox


@pytest.mark.parametrize("seed,n_views,W,H", [(1, 3, 200, 150), (5, 1, 333, 257), (2, 2, 40, 24), (4, 1, 17, 9)])
def test_tile_binning_equals_radix_sort_and_oracle(seed, n_views, W, H):
    """Small images of a many-voxel scene put thousands of records in a tile (the global-memory
    path of the per-tile sort); larger images keep tiles in shared memory."""
    sc = S.scene_small(seed=seed)
    cams = S.ring_cameras(n_views, 3.0, W, H, fovx_deg=50.0, phase=0.2 * seed)
    po = PairOrder(torch.as_tensor(sc.octpath.reshape(-1), device="cuda"))
    st_t, v_t, r_t = _bin(sc, cams, po)
    st_r, v_r, r_r = _bin(sc, cams, None)
    assert st_t.num_rendered == st_r.num_rendered > 0
    assert np.array_equal(v_t, v_r), "record order differs from the radix sort"
    assert np.array_equal(r_t, r_r)
    assert st_t.status() == 0
    counts = (r_t[:, 1] - r_t[:, 0]).astype(np.int64)
    if W * H < 2000:
        assert counts.max() > 4096, "the case is meant to exercise the large-tile path"
    # the oracle, view by view (each view's tiles are a contiguous block of the batch)
    off = 0
    for cam in cams:
        geos, rgbs = oracle_inputs(sc, cam)
        ref = oracle_view(sc, cam, geos, rgbs)
        nt = ((cam.width + 15) // 16) * ((cam.height + 15) // 16)
        rg = r_t[off:off + nt]
        nonempty = ref["ranges"][:, 1] > ref["ranges"][:, 0]
        base = rg[nonempty][0, 0] if nonempty.any() else 0
        sel = v_t[base:base + len(ref["vals"])]
        assert np.array_equal(sel, ref["vals"])
        assert np.array_equal(rg[nonempty] - base, ref["ranges"][nonempty])
        off += nt


def test_tile_binning_images_equal_radix_sort_images():
    sc = S.scene_small(seed=6)
    cams = S.ring_cameras(2, 3.0, 160, 120, fovx_deg=50.0)
    po = PairOrder(torch.as_tensor(sc.octpath.reshape(-1), device="cuda"))
    geos, _ = oracle_inputs(sc, cams[0])
    rgbs = np.concatenate([oracle_inputs(sc, c)[1] for c in cams], 0)
    ts = torch_scene(sc)
    s_val = torch.tensor([sc.s_val], dtype=torch.float32, device="cuda")
    outs = []
    for table in (po, None):
        st, _, _ = _bin(sc, cams, table)
        outs.append(st.render(3, True, True, ts["centers"], ts["lengths"], torch.as_tensor(geos).cuda(),
                              torch.as_tensor(rgbs).cuda(), s_val, rgb_per_view=True))
    for a, b in zip(outs[0][:4], outs[1][:4]):
        assert torch.equal(a, b)


def test_tile_binning_with_capacity():
    sc = S.scene_small(seed=2)
    cams = S.ring_cameras(2, 3.0, 160, 120, fovx_deg=50.0)
    po = PairOrder(torch.as_tensor(sc.octpath.reshape(-1), device="cuda"))
    st0, v0, r0 = _bin(sc, cams, po)
    st1, v1, r1 = _bin(sc, cams, po, capacity=2_000_000)
    n = st0.num_rendered
    assert st1.binned_count() == n
    assert np.array_equal(v1[:n], v0) and np.array_equal(r1, r0)
    assert st1.status() == 0
    # a capacity below the total: flagged, every range inside the capacity
    st2, _, r2 = _bin(sc, cams, po, capacity=n // 2)
    assert st2.status() & 8
    assert r2.max() <= n // 2


def test_tile_binning_mid_size_all_views_equals_radix_sort():
    """All 8 views of 800x800 of the mid-size workload (13.6M records): the per-tile sort and
    the radix sort give the same record order and tile ranges."""
    import bench
    sc, cams = bench.make_workload(0, config="mid")
    po = PairOrder(torch.as_tensor(sc.octpath.reshape(-1), device="cuda"))
    st_t, v_t, r_t = _bin(sc, cams, po)
    st_r, v_r, r_r = _bin(sc, cams, None)
    assert st_t.num_rendered == st_r.num_rendered > 10_000_000
    assert np.array_equal(r_t, r_r)
    assert np.array_equal(v_t, v_r)
    assert st_t.status() == 0


@pytest.mark.parametrize("key_bits", [24, 28, 32])
def test_tile_sort_paths_for_wider_keys(key_bits):
    """The same pair positions declared with more key bits move the large tiles' top-digit
    split onto high (mostly zero) bits: one-bucket splits, second-level splits and, at 32 bits,
    buckets of more than one block-tile sorted by passes over global memory.  The record order
    must stay that of the radix sort."""
    from types import SimpleNamespace
    sc = S.scene_small(seed=2)
    cams = S.ring_cameras(2, 3.0, 40, 24, fovx_deg=50.0, phase=0.4)
    po = PairOrder(torch.as_tensor(sc.octpath.reshape(-1), device="cuda"))
    assert key_bits >= po.bits
    wide = SimpleNamespace(pos=po.pos, bits=key_bits, N=po.N)
    st_t, v_t, r_t = _bin(sc, cams, wide)
    st_r, v_r, r_r = _bin(sc, cams, None)
    counts = (r_t[:, 1] - r_t[:, 0]).astype(np.int64)
    assert counts.max() > 4096
    assert np.array_equal(v_t, v_r) and np.array_equal(r_t, r_r)
    assert st_t.status() == 0
