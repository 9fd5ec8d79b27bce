"""Record order of the binning sort, restated on the CPU (oracle = the C restatement of
forward.cu:749-829 + stable sort):

* the records emitted in voxel-major, octant, row, column order and stably sorted by the
  full (tile, rank) key are the oracle's sorted keys and values, bit for bit;
* a stable sort by the tile bits alone followed by a stable sort of each tile's records by
  rank gives the same order (stable composition: lexicographic order with emission-order
  ties), the property a two-level sort (tile passes, then one block per tile) relies on;
* dense ranks (the sorted distinct ranks renumbered 0, 1, ...) order and tie exactly as the
  48-bit ranks do;
* so do the trimmed ranks of the binning key (``raster.rank_shift``).
"""
import numpy as np

from tests.helpers import scene_and_cams

TILE = 16
RANK_BITS = 48


def rep3(q):
    v = 0
    for _ in range(16):
        v = (v << 3) | q
    return v


def emit(cam, octpath, ndup, bb, bits):
    """The duplicate step: one (key, value) per (octant, tile) of every rendered voxel."""
    gx, gy = (cam.width + TILE - 1) // TILE, (cam.height + TILE - 1) // TILE
    keys, vals = [], []
    for i in np.flatnonzero(ndup > 0):
        b0, b1 = int(bb[i, 0]), int(bb[i, 1])
        tx0 = max(0, min(gx - 1, (b0 >> 16) // TILE)); ty0 = max(0, min(gy - 1, (b0 & 0xFFFF) // TILE))
        tx1 = max(0, min(gx - 1, (b1 >> 16) // TILE)); ty1 = max(0, min(gy - 1, (b1 & 0xFFFF) // TILE))
        path = int(octpath[i])
        for q in range(8):
            if not (int(bits[i]) >> q) & 1:
                continue
            rank = path ^ rep3(q)
            for y in range(ty0, ty1 + 1):
                for x in range(tx0, tx1 + 1):
                    keys.append(((y * gx + x) << RANK_BITS) | rank)
                    vals.append((q << 29) | int(i))
    return np.array(keys, np.uint64), np.array(vals, np.uint32)


def two_level_order(keys):
    tiles = keys >> np.uint64(RANK_BITS)
    ranks = keys & np.uint64((1 << RANK_BITS) - 1)
    by_tile = np.argsort(tiles, kind="stable")
    out = np.empty_like(by_tile)
    t_sorted = tiles[by_tile]
    starts = np.flatnonzero(np.r_[True, t_sorted[1:] != t_sorted[:-1]])
    ends = np.r_[starts[1:], len(t_sorted)]
    for s, e in zip(starts, ends):
        seg = by_tile[s:e]
        out[s:e] = seg[np.argsort(ranks[seg], kind="stable")]
    return out


def test_sort_composition_matches_the_oracle_order():
    from oracle import oracle as O
    sc, cams = scene_and_cams("small", 2, 96, 80)
    checked = 0
    for cam in cams:
        ndup, bb, bits = O.preprocess(cam, sc.vox_center, sc.vox_size, sc.is_leaf)
        okeys, ovals, _ = O.binning(cam, sc.octpath, ndup, bb, bits)
        keys, vals = emit(cam, np.asarray(sc.octpath).reshape(-1), ndup, bb, bits)
        assert len(keys) == len(okeys) == int(ndup.sum()) > 0
        one = np.argsort(keys, kind="stable")
        assert np.array_equal(keys[one], okeys) and np.array_equal(vals[one], ovals)
        two = two_level_order(keys)
        assert np.array_equal(one, two)
        # dense ranks: same order, same ties
        ranks = keys & np.uint64((1 << RANK_BITS) - 1)
        uniq, dense = np.unique(ranks, return_inverse=True)
        dkeys = ((keys >> np.uint64(RANK_BITS)) << np.uint64(32)) | dense.astype(np.uint64)
        assert np.array_equal(np.argsort(dkeys, kind="stable"), one)
        checked += len(keys)
    assert checked > 1000


def test_trimmed_rank_keeps_order_and_ties():
    """raster.rank_shift drops the low 3-bit level groups that are zero in every path but
    one: the kept group still carries the octant, so the trimmed ranks order and tie the
    (voxel, octant) pairs exactly as the full 48-bit ranks do."""
    from svraster_b200.raster import rank_shift
    rng = np.random.default_rng(3)
    for max_level in (1, 4, 9, 10, 15, 16):
        zero_groups = 16 - max_level
        paths = rng.integers(0, 1 << (3 * max_level), size=300, dtype=np.int64).astype(np.uint64)
        paths <<= np.uint64(3 * zero_groups)
        paths[:20] = paths[20:40]                        # repeated paths give ties
        path_or = int(np.bitwise_or.reduce(paths))
        shift = rank_shift(path_or)
        assert shift == (3 * (zero_groups - 1) if zero_groups > 0 else 0) or path_or & (7 << (3 * zero_groups)) == 0
        q = rng.integers(0, 8, size=paths.size)
        full = paths ^ np.array([rep3(int(x)) for x in q], np.uint64)
        trimmed = full >> np.uint64(shift)
        assert np.array_equal(np.argsort(full, kind="stable"), np.argsort(trimmed, kind="stable"))
        assert np.array_equal(full[:, None] == full[None, :], trimmed[:, None] == trimmed[None, :])
