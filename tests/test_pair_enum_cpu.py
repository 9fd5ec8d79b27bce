"""Lane-level restatement, on the CPU, of how the pair forward kernel numbers a warp's
candidate pairs (svraster_b200/csrc/render_pairs.cuh): per-lane 128-bit candidate masks, an
exclusive prefix of their counts, the owner lane of pair i found by a five-step binary search
over shuffled prefixes, the k-th set bit of the owner's mask.  Every (lane, record) candidate
must come out exactly once, lanes in order and each lane's records ascending, which is the
order the compositing phase pops them in."""
import numpy as np
import pytest


def kth_set_bit(w, k):
    pos = 0
    for s in (16, 8, 4, 2, 1):
        c = bin(w & ((1 << s) - 1)).count("1")
        if k >= c:
            k -= c
            w >>= s
            pos += s
    return pos


def enumerate_pairs(masks):
    """masks: 32 lists of 4 uint32 words -> [(lane, record)] in pair-index order."""
    cnt = [sum(bin(w).count("1") for w in m) for m in masks]
    pre = list(np.cumsum([0] + cnt[:-1]))
    total = sum(cnt)
    out = []
    for i in range(total):
        ol = 0
        for step in (16, 8, 4, 2, 1):
            cand = ol + step
            if pre[cand] <= i:
                ol = cand
        k = i - pre[ol]
        om = masks[ol]
        jb, wsel = 0, om[0]
        c = bin(om[0]).count("1")
        if k >= c:
            k -= c; wsel = om[1]; jb = 32; c = bin(om[1]).count("1")
            if k >= c:
                k -= c; wsel = om[2]; jb = 64; c = bin(om[2]).count("1")
                if k >= c:
                    k -= c; wsel = om[3]; jb = 96
        out.append((ol, jb + kth_set_bit(wsel, k)))
    return out


@pytest.mark.parametrize("density,seed", [(0.0, 0), (0.01, 1), (0.1, 2), (0.5, 3), (1.0, 4)])
def test_pairs_enumerate_every_candidate_in_order(density, seed):
    rng = np.random.default_rng(seed)
    bits = rng.random((32, 128)) < density
    bits[rng.random(32) < 0.3] = False            # idle lanes between busy ones
    masks = [[int(sum(1 << b for b in range(32) if bits[l, 32 * w + b])) for w in range(4)] for l in range(32)]
    got = enumerate_pairs(masks)
    want = [(l, j) for l in range(32) for j in range(128) if bits[l, j]]
    assert got == want


def test_kth_set_bit_all_positions():
    rng = np.random.default_rng(7)
    for _ in range(200):
        w = int(rng.integers(1, 1 << 32))
        pos = [b for b in range(32) if w >> b & 1]
        assert [kth_set_bit(w, k) for k in range(len(pos))] == pos
