"""Lane-level restatement, on the CPU, of the per-tile sort's index arithmetic
(svraster_b200/csrc/tile_sort.cuh): warp-striped block-tiles of TS_THREADS x TS_K keys, digit
peers from eight ballots, per-warp running digit counts, the block scan of the digit totals
and the chunked passes of a tile larger than one block-tile.  Checks that the positions it
computes sort any key set exactly (keys unique, as pair positions are) and stay in range, and
that the launch-bucket order of the tile scan is heavy first and stable."""
import numpy as np
import pytest

THREADS, K = 256, 16
WARPS = THREADS // 32
CHUNK = THREADS * K


def digit_peers(d, valid):
    """[32] digits, [32] valid -> [32] peer masks as the eight-ballot AND computes them."""
    lanes = np.arange(32)
    ballot = lambda pred: int(np.sum(np.where(pred, 1 << lanes, 0)))
    peers = np.full(32, ballot(valid), dtype=np.int64)
    for b in range(8):
        bit = (d >> b) & 1
        bal = ballot(bit == 1)
        peers &= np.where(bit == 1, bal, ~bal & 0xFFFFFFFF)
    return peers


def block_rank(keys_bt, count, sh, base):
    """keys_bt[WARPS, K, 32] of one block-tile; returns destination positions like the kernel
    (base: None = exclusive scan of the block-tile's own digit totals, else running base)."""
    whist = np.zeros((WARPS, 256), np.int64)
    pos = np.zeros((WARPS, K, 32), np.int64)
    lt = [(1 << l) - 1 for l in range(32)]
    for w in range(WARPS):
        for k in range(K):
            i = w * 32 * K + k * 32 + np.arange(32)
            valid = i < count
            d = (keys_bt[w, k] >> sh) & 255
            peers = digit_peers(d, valid)
            before = np.where(valid, whist[w, d], 0)
            pos[w, k] = before + np.array([bin(int(peers[l]) & lt[l]).count("1") for l in range(32)])
            for l in range(32):
                if valid[l] and l == int(peers[l]).bit_length() - 1:
                    whist[w, d[l]] = before[l] + bin(int(peers[l])).count("1")
    tot = whist.sum(0)
    run = (np.concatenate([[0], np.cumsum(tot)[:-1]]) if base is None else base.copy())
    if base is not None:
        base += tot
    wbase = np.zeros_like(whist)
    for w in range(WARPS):
        wbase[w] = run
        run = run + whist[w]
    for w in range(WARPS):
        for k in range(K):
            d = (keys_bt[w, k] >> sh) & 255
            pos[w, k] += wbase[w, d]
    return pos


def striped(arr, c0, cnt):
    out = np.zeros((WARPS, K, 32), np.int64)
    for w in range(WARPS):
        for k in range(K):
            i = w * 32 * K + k * 32 + np.arange(32)
            ok = i < cnt
            out[w, k, ok] = arr[c0 + i[ok]]
    return out


def tile_sort(keys, key_bits):
    """The kernel's two paths on one tile; returns the keys in their final order."""
    n = len(keys)
    npass = (key_bits + 7) // 8
    src = keys.astype(np.int64).copy()
    for p in range(npass):
        sh = 8 * p
        dst = np.full(n, -1, np.int64)
        if n <= CHUNK:
            kb = striped(src, 0, n)
            pos = block_rank(kb, n, sh, None)
            for w in range(WARPS):
                for k in range(K):
                    i = w * 32 * K + k * 32 + np.arange(32)
                    ok = i < n
                    assert np.all(pos[w, k, ok] < n)
                    dst[pos[w, k, ok]] = kb[w, k, ok]
        else:
            hist = np.bincount((src >> sh) & 255, minlength=256)
            base = np.concatenate([[0], np.cumsum(hist)[:-1]])
            for c0 in range(0, n, CHUNK):
                cnt = min(CHUNK, n - c0)
                kb = striped(src, c0, cnt)
                pos = block_rank(kb, cnt, sh, base)
                for w in range(WARPS):
                    for k in range(K):
                        i = w * 32 * K + k * 32 + np.arange(32)
                        ok = i < cnt
                        assert np.all(pos[w, k, ok] < n)
                        dst[pos[w, k, ok]] = kb[w, k, ok]
        assert np.all(dst >= 0), "a position was written twice or never"
        src = dst
    return src


@pytest.mark.parametrize("n,key_bits,seed", [(1, 8, 0), (37, 12, 1), (4096, 24, 2), (3000, 26, 3),
                                             (4097, 24, 4), (9000, 26, 5)])
def test_tile_sort_positions_sort_unique_keys(n, key_bits, seed):
    rng = np.random.default_rng(seed)
    keys = rng.choice(1 << key_bits, size=n, replace=False)
    out = tile_sort(keys, key_bits)
    assert np.array_equal(out, np.sort(keys))


def heavy_bucket(c):
    if c == 0:
        return 255
    e = c.bit_length() - 1
    m = (c >> (e - 3)) & 7 if e >= 3 else (c << (3 - e)) & 7
    return 254 - min(e * 8 + m, 254)


def test_launch_buckets_heavy_first_and_monotone():
    counts = [0, 1, 2, 3, 7, 8, 9, 15, 16, 100, 1000, 4095, 4096, 72000, 1 << 20, (1 << 31) + 5]
    b = [heavy_bucket(c) for c in counts]
    assert all(0 <= x <= 255 for x in b)
    assert b[0] == 255
    assert all(b[i] >= b[i + 1] for i in range(1, len(b) - 1))   # more records, earlier bucket
    rng = np.random.default_rng(0)
    c = rng.integers(0, 80000, size=5000)
    order = sorted(range(len(c)), key=lambda t: (heavy_bucket(int(c[t])), t))
    assert all(heavy_bucket(int(c[order[i]])) <= heavy_bucket(int(c[order[i + 1]])) for i in range(len(c) - 1))
