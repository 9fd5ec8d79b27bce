"""Capacity-mode binning (no host read-back of the record total) and the CUDA-graph-captured
training step: same images, binning and gradients as the eager step, status words flag a
capacity overflow, and the step counter drives the Adam coefficients and smoothness jitter
on every replay."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from svraster_b200 import synthetic as S
from svraster_b200.raster import RasterState
from svraster_b200.step import BatchedTrainStep
from tests.helpers import scene_and_cams

pytestmark = pytest.mark.gpu


def _tensors(sc, dev):
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    return (t(sc.octpath, torch.int64), t(sc.vox_center), t(sc.vox_size).reshape(-1).contiguous(),
            t(sc.is_leaf, torch.uint8))


def _views(cams, dev):
    return [dict(width=c.width, height=c.height, tanfovx=c.tanfovx, tanfovy=c.tanfovy, cx=c.cx, cy=c.cy,
                 near=c.near, w2c=torch.as_tensor(c.w2c).to(dev), c2w=torch.as_tensor(c.c2w).to(dev),
                 bg=torch.zeros(3, device=dev)) for c in cams]


def _render(sc, cams, dev, capacity=None, path_or=None):
    octpath, centers, lengths, is_leaf = _tensors(sc, dev)
    st = RasterState(_views(cams, dev), sc.n_vox, dev)
    st.preprocess(octpath, centers, lengths, is_leaf)
    st.bin(octpath, capacity=capacity, path_or=path_or)
    g = torch.Generator().manual_seed(3)
    geos = torch.as_tensor(sc.geo_grid_pts[sc.vox_key].reshape(-1, 8)).to(dev).contiguous()
    rgbs = torch.rand(sc.n_vox, 3, generator=g).to(dev)
    s_val = torch.tensor([sc.s_val], dtype=torch.float32, device=dev)
    color, depth, normal, T, _ = st.render(3, True, True, centers, lengths, geos, rgbs, s_val)
    torch.cuda.synchronize()
    return st, color.cpu(), depth.cpu(), T.cpu()


def _path_or_all(sc):
    p = np.asarray(sc.octpath, np.int64)[np.asarray(sc.is_leaf).astype(bool).reshape(-1)]
    return int(np.bitwise_or.reduce(p.view(np.uint64)))


@pytest.mark.parametrize("extra", [0, 777])
def test_capacity_binning_matches_exact_count(extra):
    dev = torch.device("cuda")
    sc, cams = scene_and_cams("small", n_cams=3, W=160, H=120)
    ref, c0, d0, T0 = _render(sc, cams, dev)
    R = ref.num_rendered
    cap, c1, d1, T1 = _render(sc, cams, dev, capacity=R + extra, path_or=_path_or_all(sc))
    assert cap.binned_count() == R
    assert cap.status() == 0
    v0, r0, tl0, nc0 = ref.binning_fields()
    v1, r1, tl1, nc1 = cap.binning_fields()
    assert torch.equal(v0.cpu(), v1[:R].cpu())
    assert torch.equal(r0.cpu(), r1.cpu()) and torch.equal(tl0.cpu(), tl1.cpu()) and torch.equal(nc0.cpu(), nc1.cpu())
    assert torch.equal(c0, c1) and torch.equal(d0, d1) and torch.equal(T0, T1)


def test_record_packing_sources_agree():
    """Record packing takes centre and length from a per-voxel float4 when the record
    capacity is at least twice the voxel count, and from the two arrays otherwise: the same
    records either way, so the same binning and images, bit for bit."""
    dev = torch.device("cuda")
    sc, cams = scene_and_cams("small", n_cams=1, W=160, H=120)
    ref, c0, d0, T0 = _render(sc, cams, dev)
    R = ref.num_rendered
    assert 0 < R < 2 * sc.n_vox                      # exact count: the two-array source
    cap, c1, d1, T1 = _render(sc, cams, dev, capacity=2 * sc.n_vox + 5, path_or=_path_or_all(sc))
    assert cap.binned_count() == R and cap.status() == 0
    v0, r0, _, _ = ref.binning_fields()
    v1, r1, _, _ = cap.binning_fields()
    assert torch.equal(v0.cpu(), v1[:R].cpu()) and torch.equal(r0.cpu(), r1.cpu())
    assert torch.equal(c0, c1) and torch.equal(d0, d1) and torch.equal(T0, T1)


def test_capacity_overflow_is_flagged_not_faulted():
    dev = torch.device("cuda")
    sc, cams = scene_and_cams("small", n_cams=2, W=128, H=96)
    ref, *_ = _render(sc, cams, dev)
    R = ref.num_rendered
    cap, *_ = _render(sc, cams, dev, capacity=R // 2, path_or=_path_or_all(sc))
    assert cap.binned_count() == R // 2
    assert cap.status() & 8


def test_key_format_violation_is_flagged():
    dev = torch.device("cuda")
    sc, cams = scene_and_cams("small", n_cams=1, W=128, H=96)
    ref, *_ = _render(sc, cams, dev)
    # a path_or with only the top level set trims bits the rendered paths do use
    top = 7 << 45
    bad, *_ = _render(sc, cams, dev, capacity=ref.num_rendered, path_or=top)
    assert bad.status() & 16


def _step_pair(lambda_ls=1e-2, lambda_ge=1e-2):
    sc = S.scene_small(seed=2)
    cams = S.fibonacci_cameras(3, 3.0, 144, 112, fovx_deg=50.0)
    a = BatchedTrainStep(sc, cams, device="cuda", lambda_ls=lambda_ls, lambda_ge=lambda_ge, lambda_R_concen=0.1)
    b = BatchedTrainStep(sc, cams, device="cuda", lambda_ls=lambda_ls, lambda_ge=lambda_ge, lambda_R_concen=0.1)
    return a, b


def _param_close(pa, pb, lr):
    d = (pa - pb).abs()
    # float atomics in the adjoint make the gradients order-dependent in the last bits; Adam
    # with eps 1e-15 maps a sign flip of a vanishing gradient to a 2*lr change, so allow a
    # small fraction of such elements
    bad = (d > 1e-6).float().mean().item()
    return bad < 2e-3 and d.max().item() <= 2.5 * lr


def test_graph_replay_matches_eager_steps():
    a, b = _step_pair()
    n = b.capture()
    assert n >= 10
    for k in range(3):
        ca, Ta = a.step()
        cb, Tb = b.replay()
        torch.cuda.synchronize()
        if k == 0:
            # same parameters in, deterministic forward: images agree bit for bit
            assert torch.equal(ca, cb) and torch.equal(Ta, Tb)
    assert int(b.step_dev.item()) == 3 and b.adam_step == 3
    assert b.graph_status() == (0, 0)
    for pa, pb, lr in zip(a.params, b.params, a.lr):
        assert _param_close(pa, pb, lr)


def test_graph_replay_advances_jitter_seed():
    """With the smoothness adjoints alone driving Adam on untouched grid points, a replay
    that reused the captured seed would drift from the eager steps (seed + step)."""
    a, b = _step_pair(lambda_ls=1.0, lambda_ge=1.0)
    b.capture()
    for _ in range(2):
        a.step()
        b.replay()
    torch.cuda.synchronize()
    assert _param_close(a.grid, b.grid, a.lr[0])


def test_eager_step_after_replays_resyncs_counter():
    a, b = _step_pair()
    b.capture()
    b.replay()
    b.step()            # eager step 2 on the host counter
    b.replay()          # replay must run as step 3
    for _ in range(3):
        a.step()
    torch.cuda.synchronize()
    assert int(b.step_dev.item()) == 3
    for pa, pb, lr in zip(a.params, b.params, a.lr):
        assert _param_close(pa, pb, lr)


def test_bf16_sh_step_eager_and_replay():
    """SH coefficients stored in bf16: the step keeps them bf16, replay equals eager, and the
    first image stays within the bf16 storage step of the f32 step's image."""
    sc = S.scene_small(seed=2)
    cams = S.fibonacci_cameras(3, 3.0, 144, 112, fovx_deg=50.0)
    a = BatchedTrainStep(sc, cams, device="cuda", lambda_R_concen=0.1, sh_dtype="bf16")
    b = BatchedTrainStep(sc, cams, device="cuda", lambda_R_concen=0.1, sh_dtype="bf16")
    f = BatchedTrainStep(sc, cams, device="cuda", lambda_R_concen=0.1)
    b.capture()
    ca, _ = a.step()
    cb, _ = b.replay()
    cf, _ = f.step()
    torch.cuda.synchronize()
    assert a.sh0.dtype == torch.bfloat16 and a.shs.dtype == torch.bfloat16
    assert torch.equal(ca, cb)
    assert (ca - cf).abs().max().item() < 2e-2
    for _ in range(2):
        a.step()
        b.replay()
    torch.cuda.synchronize()
    assert b.graph_status() == (0, 0)
    assert _param_close(a.grid, b.grid, a.lr[0])
    d = (a.sh0.float() - b.sh0.float()).abs()
    assert (d > 0).float().mean().item() < 2e-3


def test_split_capture_matches_whole_capture():
    """capture(split=True): the forward and backward graphs replayed in turn give the same
    images and (up to atomic order) the same parameters as the whole-step graph, and the
    backward graph reads the upstream planes as they are when it runs."""
    a, b = _step_pair()
    a.capture()
    b.capture(split=True)
    for k in range(2):
        ca, Ta = a.replay()
        b.replay_forward()
        cb, Tb = b.replay_backward()
        torch.cuda.synchronize()
        if k == 0:
            assert torch.equal(ca, cb) and torch.equal(Ta, Tb)
    assert a.adam_step == b.adam_step == 2
    assert b.graph_status() == (0, 0)
    for pa, pb, lr in zip(a.params, b.params, a.lr):
        assert _param_close(pa, pb, lr)
    # upstream planes rewritten between the two parts are what that step's adjoint reads:
    # zeroing them there equals an eager step with zeroed planes
    c, d = _step_pair()
    c.capture(split=True)
    c.replay_forward()
    for x in (c.dcolor, c.ddepth, c.dnormal):
        x.zero_()
    c.replay_backward()
    for x in (d.dcolor, d.ddepth, d.dnormal):
        x.zero_()
    d.step()
    torch.cuda.synchronize()
    for pc, pd, lr in zip(c.params, d.params, c.lr):
        assert _param_close(pc, pd, lr)


def test_split_capture_with_two_upstream_sets():
    """upstream_sets=2: the second backward graph reads the second plane set; alternating sets
    that hold the same planes gives the single-set result."""
    a, b = _step_pair()
    a.capture(split=True)
    b.capture(split=True, upstream_sets=2)
    for x, y in zip(b.upstream(0), b.upstream(1)):
        assert x is not y and (x is None or torch.equal(x, y))
    for k in range(3):
        a.replay_forward()
        ca, Ta = a.replay_backward()
        b.replay_forward()
        cb, Tb = b.replay_backward(k % 2)
        torch.cuda.synchronize()
        if k == 0:
            assert torch.equal(ca, cb) and torch.equal(Ta, Tb)
    assert b.graph_status() == (0, 0)
    for pa, pb, lr in zip(a.params, b.params, a.lr):
        assert _param_close(pa, pb, lr)
