"""Lane-level restatement of two device helpers of the fused smoothness adjoint
(svraster_b200/csrc/grid_loss.cu), checked on the CPU:

* ``run_sum8``: the segmented shuffle reduction that sums each run of lanes holding the
  same primary voxel into the run's head lane stops after the rounds the warp's longest
  run needs.  The heads' float32 sums must be bit-identical to the ones all five rounds
  give (the GPU-side comparison against the separate Laplacian / Eikonal kernels is
  tests/test_gpu_smoothness_fused.py).
* ``clamp01``: the NaN-propagating max/min pair equals the compare-and-assign clamp of the
  trilinear weights for every input except -0.0.
"""
import numpy as np


def _shuffle_rounds(primary, acc, rounds):
    """The device loop: for off = 1, 2, 4, ... (``rounds`` of them) every lane adds the value
    of lane + off when that lane is in the same run.  Returns the lanes' sums."""
    lanes = len(primary)
    head = np.array([i == 0 or primary[i - 1] != primary[i] for i in range(lanes)])
    heads_idx = np.flatnonzero(head)
    my_head = np.array([heads_idx[heads_idx <= i].max() for i in range(lanes)])
    a = acc.copy()
    off = 1
    for _ in range(rounds):
        nxt = a.copy()
        for i in range(lanes):
            j = i + off
            if j < lanes and my_head[j] == my_head[i]:
                nxt[i] = np.float32(a[i] + a[j])
        a = nxt
        off <<= 1
    return a, head


def _longest_run_rounds(primary):
    lanes = len(primary)
    head = [i == 0 or primary[i - 1] != primary[i] for i in range(lanes)]
    runs, start = [], 0
    for i in range(1, lanes + 1):
        if i == lanes or head[i]:
            runs.append(i - start)
            start = i
    longest = max(runs)
    rounds, off = 0, 1
    while off < longest:          # for (off = 1; off < longest; off <<= 1)
        rounds += 1
        off <<= 1
    return rounds


def test_run_sum_stops_at_longest_run_with_identical_head_sums():
    rng = np.random.default_rng(11)
    for trial in range(400):
        # runs of random lengths (1..32) of equal primaries, -1 for lanes without a sample
        lengths = []
        while sum(lengths) < 32:
            lengths.append(int(rng.integers(1, 33 if trial % 4 == 0 else 6)))
        primary, v = [], 0
        for n in lengths:
            primary += [v if rng.random() > 0.1 else -1] * n
            v += 1
        primary = np.array(primary[:32])
        acc = rng.normal(size=(32, 8)).astype(np.float32) * np.float32(10.0) ** rng.integers(-3, 4, size=(32, 1))
        full, head = _shuffle_rounds(primary, acc, 5)
        short, _ = _shuffle_rounds(primary, acc, _longest_run_rounds(primary))
        assert np.array_equal(full[head].view(np.uint32), short[head].view(np.uint32))


def test_single_lane_runs_need_no_rounds():
    assert _longest_run_rounds(np.arange(32)) == 0
    assert _longest_run_rounds(np.zeros(32, dtype=int)) == 5
    assert _longest_run_rounds(np.array([0, 0, 0] + list(range(1, 30)))) == 2


def _clamp_compare(w):
    w = w.copy()
    w[w < 0] = 0
    w[w > 1] = 1
    return w


def _clamp_nan_minmax(w):
    # max.NaN / min.NaN: a NaN operand gives NaN; otherwise the ordinary max / min
    return np.minimum(np.maximum(w, np.float32(0)), np.float32(1))


def test_weight_clamp_matches_except_negative_zero():
    rng = np.random.default_rng(5)
    w = np.concatenate([rng.normal(size=10000).astype(np.float32),
                        np.array([0.0, 1.0, -1e-45, 1e-45, 1.0000001, np.inf, -np.inf, np.nan], np.float32)])
    a, b = _clamp_compare(w), _clamp_nan_minmax(w)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    finite = ~np.isnan(a)
    assert np.array_equal(a[finite].view(np.uint32), b[finite].view(np.uint32))
    # -0.0: kept by the compare form, +0.0 from the max (a zero weight either way)
    nz = np.array([-0.0], np.float32)
    assert _clamp_compare(nz)[0] == 0 and _clamp_nan_minmax(nz)[0] == 0
