"""The fused per-voxel smoothness adjoint (svr_smoothness_bw_vox followed by the per-voxel
gradient scatter) against the separate Laplacian and grid-Eikonal adjoints with the same
seed: equal up to the order of the floating-point additions."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from svraster_b200 import _lib
from svraster_b200 import synthetic as S
from svraster_b200._lib import check, ptr, stream_ptr
from svraster_b200.step import BatchedTrainStep

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def step():
    sc = S.scene_small(seed=5)
    cams = S.fibonacci_cameras(2, 3.0, 64, 48, fovx_deg=50.0)
    st = BatchedTrainStep(sc, cams, device="cuda")
    L = _lib.load()
    check(L.svr_gather_geo(st.N, ptr(st.all_idx), ptr(st.vox_key), ptr(st.grid), ptr(st.geos),
                           stream_ptr(st.dev)), "gather")
    return st


def _separate(st, w_ls, w_ge, seed, active):
    L = _lib.load()
    grad = torch.zeros_like(st.grid)
    status = torch.zeros(1, dtype=torch.int32, device=st.dev)
    G, A = st.grid_keys.numel(), active.numel()
    for fn, lam in ((L.svr_laplacian_bw, w_ls), (L.svr_eikonal_bw, w_ge)):
        if lam == 0:
            continue
        check(fn(G, A, ptr(active), ptr(st.grid_keys), ptr(st.grid2voxel), 1 << st.res_pow2, ptr(st.grid_mask),
                 ptr(st.grid_index), ptr(st.grid_voxel_coord), ptr(st.grid_voxel_size), st.N, ptr(st.vox_key),
                 ptr(st.grid), st.grid.numel(), float(lam), st.vox_size_min_inv, seed, ptr(grad), ptr(status),
                 stream_ptr(st.dev)), "separate")
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return grad


def _fused(st, w_ls, w_ge, seed, active, seed_step=None):
    L = _lib.load()
    dvox = torch.zeros(st.N, 12, device=st.dev)
    grad = torch.zeros_like(st.grid)
    status = torch.zeros(1, dtype=torch.int32, device=st.dev)
    G = st.grid_keys.numel()
    A = G if active is None else active.numel()
    check(L.svr_smoothness_bw_vox(G, A, ptr(active), ptr(st.grid_keys), ptr(st.grid2voxel), 1 << st.res_pow2,
                                  ptr(st.grid_mask), ptr(st.grid_index), ptr(st.grid_voxel_coord),
                                  ptr(st.grid_voxel_size), st.N, ptr(st.geos), float(w_ls), float(w_ge),
                                  st.vox_size_min_inv, seed, ptr(seed_step), ptr(dvox), 12, ptr(status),
                                  stream_ptr(st.dev)), "fused")
    check(L.svr_scatter_vox_grads(st.N, 12, ptr(st.vox_key), ptr(dvox), ptr(grad), stream_ptr(st.dev)), "scatter")
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert torch.count_nonzero(dvox[:, 8:]) == 0
    return grad


def _close(a, b):
    scale = b.abs().max().item()
    assert scale > 0
    err = (a - b).abs().max().item()
    assert err <= 1e-5 * scale, (err, scale)


@pytest.mark.parametrize("w_ls,w_ge", [(1e-2, 1e-2), (1e-2, 0.0), (0.0, 1e-2), (1.0, 3e-3)])
def test_fused_equals_separate_all_keys(step, w_ls, w_ge):
    G = step.grid_keys.numel()
    all_rows = torch.arange(G, dtype=torch.int32, device=step.dev)
    _close(_fused(step, w_ls, w_ge, 11, None), _separate(step, w_ls, w_ge, 11, all_rows))


def test_fused_equals_separate_random_subset(step):
    # the reference trains with active_list = randperm(G)[:K]
    G = step.grid_keys.numel()
    g = torch.Generator().manual_seed(0)
    active = torch.randperm(G, generator=g)[: G // 2].to(torch.int32).to(step.dev)
    _close(_fused(step, 1e-2, 1e-2, 4, active), _separate(step, 1e-2, 1e-2, 4, active))


def test_fused_seed_from_device_counter(step):
    counter = torch.tensor([5], dtype=torch.int64, device=step.dev)
    a = _fused(step, 1e-2, 1e-2, 2, None, seed_step=counter)
    b = _fused(step, 1e-2, 1e-2, 7, None)
    _close(a, b)
