"""Lane-level restatement, on the CPU, of the per-tile sort's index arithmetic
(svraster_b200/csrc/tile_sort.cuh): warp-striped block-tiles of TS_THREADS x TS_K keys, digit
peers from eight ballots, per-warp running digit counts, the block scan of the digit totals
and the chunked passes over global memory; and the large-tile path (top-digit split, runs of
buckets sorted over the bits they span, second split, global fallback).  Checks that the
positions it computes sort any key set exactly (keys unique, as pair positions are) and stay
in range, and that the launch-bucket order of the tile scan is heavy first and stable."""
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


def _lsd_bits_suffice(keys, kbase, npass):
    """The in-shared-memory and global LSD sorts order by the low 8 * npass bits of key - kbase:
    exact iff every key of the run is in [kbase, kbase + 2^(8 npass))."""
    rel = keys.astype(np.int64) - kbase
    return bool(np.all(rel >= 0) and np.all(rel < (1 << (8 * npass))))


def large_tile_sort(keys, key_bits, rng):
    """Restatement of the large-tile path (msd_split, sort_buckets, lsd_global): split on the
    top 8 key bits in an arbitrary order inside each bucket, runs of consecutive buckets of at
    most CHUNK records sorted by their LSD passes (checked to cover the run's keys), a bucket
    above CHUNK split again on the next 8 bits, and past two splits sorted by global passes.
    Returns the final order and the path counters."""
    out = np.full(len(keys), -1, np.int64)
    stats = {"runs": 0, "level2": 0, "global": 0}

    def split(seg, sh):
        d = (seg >> sh) & 255
        cnt = np.bincount(d, minlength=256)
        off = np.concatenate([[0], np.cumsum(cnt)[:-1]])
        res = np.empty_like(seg)
        for b in range(256):
            part = seg[d == b]
            res[off[b]:off[b] + cnt[b]] = rng.permutation(part)   # unordered within a bucket
        return res, cnt, off

    def buckets(seg, start, sh, prefix, cnt, off, level):
        b = 0
        while b < 256:
            c = int(cnt[b])
            if c == 0:
                b += 1
                continue
            o = int(off[b])
            if c > CHUNK:
                sub = seg[o:o + c]
                if level == 0 and sh > 0:
                    sh2 = max(sh - 8, 0)
                    sseg, scnt, soff = split(sub, sh2)
                    stats["level2"] += 1
                    buckets(sseg, start + o, sh2, prefix | (b << sh), scnt, soff, 1)
                else:
                    npass = max(1, (sh + 7) // 8)
                    # global passes order by the low 8*npass bits; the bucket's keys share the rest
                    assert _lsd_bits_suffice(sub, prefix | (b << sh), npass)
                    out[start + o:start + o + c] = np.sort(sub)
                    stats["global"] += 1
                b += 1
                continue
            e, last, total = b + 1, b, c
            while e < 256:
                ce = int(cnt[e])
                if ce > CHUNK or total + ce > CHUNK:
                    break
                if ce:
                    total += ce
                    last = e
                e += 1
            span = ((last - b + 1) << sh) - 1
            npass = max(1, (span.bit_length() + 7) // 8)
            run = seg[o:o + total]
            assert _lsd_bits_suffice(run, prefix | (b << sh), npass)
            out[start + o:start + o + total] = np.sort(run)
            stats["runs"] += 1
            b = e

    sh = max(key_bits - 8, 0)
    seg, cnt, off = split(keys.astype(np.int64), sh)
    buckets(seg, 0, sh, 0, cnt, off, 0)
    assert np.all(out >= 0)
    return out, stats


@pytest.mark.parametrize("case", ["uniform", "clustered", "dense_wide", "one_bucket", "small_bits", "tiny_bits",
                                  "chunk_plus_1"])
def test_large_tile_split_path_sorts_exactly(case):
    rng = np.random.default_rng(7)
    if case == "uniform":
        kb, keys = 25, rng.choice(1 << 25, size=40000, replace=False)
    elif case == "clustered":      # a few dense clusters: level-2 splits
        kb = 25
        keys = np.unique(np.concatenate([rng.choice(np.arange(c, c + 9000), size=6000, replace=False)
                                         for c in (5 << 17, (5 << 17) + 40000, 200 << 17)]))
        keys = np.concatenate([keys, np.arange(100 << 17, (100 << 17) + 12000)])
    elif case == "dense_wide":     # 30-bit keys, a dense run inside one level-2 bucket: global passes
        kb = 30
        keys = np.concatenate([np.arange(3 << 22, (3 << 22) + 7000), rng.choice(1 << 30, size=3000, replace=False)])
        keys = np.unique(keys)
    elif case == "one_bucket":     # every key in one top-digit bucket
        kb, keys = 24, (7 << 16) + rng.choice(1 << 16, size=20000, replace=False)
    elif case == "small_bits":
        kb, keys = 14, rng.choice(1 << 14, size=9000, replace=False)
    elif case == "tiny_bits":
        kb, keys = 13, np.arange(1 << 13)
    else:
        kb, keys = 20, rng.choice(1 << 20, size=CHUNK + 1, replace=False)
    keys = rng.permutation(np.asarray(keys, np.int64))
    assert keys.max() < (1 << kb)
    out, stats = large_tile_sort(keys, kb, rng)
    assert np.array_equal(out, np.sort(keys))
    if case == "clustered":
        assert stats["level2"] >= 1, stats
    if case == "dense_wide":
        assert stats["level2"] >= 1 and stats["global"] >= 1, stats


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
