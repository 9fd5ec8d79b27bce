"""Index arithmetic of the candidate rows (svraster_b200/csrc/render_pairs.cuh, raster.cu),
restated on the CPU: the forward of a tile with records [r0, r1) stores the masks of its slot s
in row block r0 // 128 + tile + s; the adjoint takes its slots from the last one down and cuts
each row at the pixel's last-contributor count.  Checks that the blocks are distinct and below
the region's size R // 128 + T + 1, that the adjoint's slots cover the tile's records once,
and the four-word cut against a plain bit mask."""
import numpy as np
import pytest

BATCH = 128


def cand_slot_count(R, T):
    return max(R, 0) // BATCH + max(T, 0) + 1


def row_blocks(r0, r1, tile):
    n = r1 - r0
    return [r0 // BATCH + tile + s for s in range((n + BATCH - 1) // BATCH)]


def adjoint_slots(n):
    """(lo, cnt) of the adjoint's batches b = 0, 1, ... (back to front)."""
    nb = (n + BATCH - 1) // BATCH
    out = []
    for b in range(nb):
        lo = (nb - 1 - b) * BATCH
        out.append((lo, min(BATCH, n - lo)))
    return out


def row_cut(last_c, lo):
    """The four mask words the adjoint ANDs with the forward's row (bits r with lo + r < last_c)."""
    k = min(max(last_c - lo, 0), BATCH)
    low = lambda c: 0xFFFFFFFF if c >= 32 else (1 << c) - 1
    return [low(min(k, 32)), low(min(max(k - 32, 0), 32)), low(min(max(k - 64, 0), 32)), low(min(max(k - 96, 0), 32))]


@pytest.mark.parametrize("seed", range(6))
def test_row_blocks_are_distinct_and_in_bounds(seed):
    rng = np.random.default_rng(seed)
    T = int(rng.integers(1, 400))
    # tile sizes: many empty, many small, a few large (as on the bench scenes)
    sizes = rng.choice([0, 0, 1, 3, 50, 127, 128, 129, 700, 5000], size=T)
    if seed % 2:
        sizes = rng.integers(0, 300, size=T)
    R_used = int(sizes.sum())
    R = R_used + int(rng.integers(0, 1000))        # the binning capacity may exceed the total
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    seen = set()
    limit = cand_slot_count(R, T)
    for tile, (r0, n) in enumerate(zip(starts.tolist(), sizes.tolist())):
        for blk in row_blocks(r0, r0 + n, tile):
            assert 0 <= blk < limit
            assert blk not in seen
            seen.add(blk)


@pytest.mark.parametrize("n", [1, 5, 127, 128, 129, 255, 256, 257, 1000])
def test_adjoint_slots_cover_the_records_once_in_forward_alignment(n):
    covered = []
    prev_lo = None
    for lo, cnt in adjoint_slots(n):
        assert lo % BATCH == 0 and 1 <= cnt <= BATCH       # the forward's slot boundaries
        assert prev_lo is None or lo < prev_lo               # back to front
        prev_lo = lo
        covered += range(lo, lo + cnt)
    assert sorted(covered) == list(range(n))


def test_row_cut_matches_a_plain_bit_mask():
    for lo in range(0, 512, BATCH):
        for last_c in range(0, 700, 3):
            words = row_cut(last_c, lo)
            k = min(max(last_c - lo, 0), BATCH)
            full = (1 << k) - 1
            want = [(full >> (32 * w)) & 0xFFFFFFFF for w in range(4)]
            assert words == want, (lo, last_c)
