"""Drop-in replacement of ``svraster_cuda.grid_loss_bw`` (cuda/svraster_cuda/grid_loss_bw.py).

The functions accumulate into ``grid_pts_grad`` in place and return ``None``, as the
reference's do.  ``laplacian_smoothness`` and ``grid_eikonal`` run on the sm_100a library.
The reference seeds their jitter with the GPU clock (ls_compute.cu:43, ge_compute.cu:74);
here the seed comes from torch's host RNG unless ``seed=`` is given, so runs are
reproducible under ``torch.manual_seed``.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check, ptr, stream_ptr


_INDEX_CACHE = {}


def dense_index(grid_keys, grid_res):
    """Direct-mapped key index for ``grid_keys`` (cached per keys tensor; the table is only
    rebuilt on prune / subdivide, so the cache hits on every training step)."""
    key = (grid_keys.data_ptr(), grid_keys.numel(), int(grid_res), grid_keys._version)
    hit = _INDEX_CACHE.get(key)
    if hit is not None:
        return hit[0]
    _INDEX_CACHE.clear()
    keys = grid_keys.to(torch.int32).contiguous()
    idx = torch.empty(int(grid_res) ** 3, dtype=torch.int32, device=grid_keys.device)
    status = torch.zeros(1, dtype=torch.int32, device=grid_keys.device)
    check(_lib.load().svr_grid_index_build(keys.numel(), ptr(keys), int(grid_res), ptr(idx), ptr(status),
                                           stream_ptr(grid_keys.device)), "svr_grid_index_build")
    _INDEX_CACHE[key] = (idx, keys, grid_keys)
    return idx


_STATUS = {}


def _status(dev):
    """One status word per device for the regularisers below: their kernels OR a flag into it
    when they skip an out-of-range voxel or grid-point index.  It is zeroed when it is read."""
    st = _STATUS.get(dev)
    if st is None:
        st = _STATUS[dev] = torch.zeros(1, dtype=torch.int32, device=dev)
    return st


_ORDER_CACHE = {}


def voxel_order(vox_key, M):
    """Visit order of the voxels for the ordered regulariser kernels: ``order`` (voxels sorted
    by the grid-point index of their first corner) and its inverse ``rank``; cached per
    vox_key tensor like ``dense_index`` (rebuilt only when the octree changes)."""
    key = (vox_key.data_ptr(), vox_key.numel(), int(M), vox_key._version)
    hit = _ORDER_CACHE.get(key)
    if hit is not None:
        return hit[0], hit[1]
    _ORDER_CACHE.clear()
    L = _lib.load()
    dev = vox_key.device
    vk = vox_key.to(torch.int64).contiguous()
    N = vk.shape[0]
    nbytes = C.c_size_t(0)
    check(L.svr_voxel_order_workspace_bytes(N, C.byref(nbytes)), "svr_voxel_order_workspace_bytes")
    ws = torch.empty(max(nbytes.value, 1), dtype=torch.uint8, device=dev)
    order = torch.empty(max(N, 1), dtype=torch.int32, device=dev)
    rank = torch.empty(max(N, 1), dtype=torch.int32, device=dev)
    check(L.svr_voxel_order(N, ptr(vk), int(M), ptr(order), ptr(rank), ptr(ws), nbytes.value, ptr(_status(dev)),
                            stream_ptr(dev)), "svr_voxel_order")
    _ORDER_CACHE[key] = (order, rank, vox_key)
    return order, rank


def _seed(seed):
    if seed is None:
        seed = int(torch.randint(0, 2 ** 31 - 1, (1,)).item())
    return int(seed) & 0x7FFFFFFF


def _grid_loss(fn_name, grid_pts, vox_key, grid_voxel_coord, grid_voxel_size, grid_res, grid_mask, grid_keys,
               grid2voxel, active_list, weight, vox_size_inv, grid_pts_grad, seed, use_index=True):
    _lib.require_cuda(grid_pts, vox_key, grid_keys, grid_pts_grad)
    if not grid_pts_grad.is_contiguous() or grid_pts_grad.dtype != torch.float32:
        raise RuntimeError("grid_pts_grad must be a contiguous float32 tensor (it is updated in place)")
    dev = grid_pts.device
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    act = active_list.to(torch.int32).contiguous()
    keys = grid_keys.to(torch.int32).contiguous()
    g2v = grid2voxel.to(torch.int32).contiguous()
    coords = grid_voxel_coord.to(torch.float32).contiguous()
    sizes = grid_voxel_size.reshape(-1).to(torch.float32).contiguous()
    key = vox_key.to(torch.int64).contiguous()
    grid = grid_pts.detach().to(torch.float32).contiguous()
    mask = grid_mask.contiguous()
    didx = dense_index(grid_keys, grid_res) if use_index else None
    fn = getattr(_lib.load(), fn_name)
    check(fn(keys.numel(), act.numel(), ptr(act), ptr(keys), ptr(g2v), int(grid_res), ptr(mask), ptr(didx),
             ptr(coords), ptr(sizes), key.shape[0], ptr(key), ptr(grid), grid.numel(), float(weight),
             float(vox_size_inv), _seed(seed), ptr(grid_pts_grad), ptr(status), stream_ptr(dev)), fn_name)
    return status


def laplacian_smoothness(grid_pts, vox_key, grid_voxel_coord, grid_voxel_size, grid_res, grid_mask, grid_keys,
                         grid2voxel, active_list, weight, vox_size_inv, no_tv_s, tv_sparse, grid_pts_grad,
                         seed=None, use_index=True):
    """grid_loss_bw.py:29-32 -> ls_compute.cu:111-153."""
    assert grid_pts.shape == grid_pts_grad.shape
    assert len(vox_key.shape) == 2 and vox_key.shape[1] == 8
    _grid_loss("svr_laplacian_bw", grid_pts, vox_key, grid_voxel_coord, grid_voxel_size, grid_res, grid_mask,
               grid_keys, grid2voxel, active_list, weight, vox_size_inv, grid_pts_grad, seed, use_index)


def grid_eikonal(grid_pts, vox_key, grid_voxel_coord, grid_voxel_size, grid_res, grid_mask, grid_keys, grid2voxel,
                 active_list, weight, vox_size_inv, no_tv_s, tv_sparse, grid_pts_grad, seed=None, use_index=True):
    """grid_loss_bw.py:24-27 -> ge_compute.cu:119-160."""
    assert grid_pts.shape == grid_pts_grad.shape
    assert len(vox_key.shape) == 2 and vox_key.shape[1] == 8
    _grid_loss("svr_eikonal_bw", grid_pts, vox_key, grid_voxel_coord, grid_voxel_size, grid_res, grid_mask,
               grid_keys, grid2voxel, active_list, weight, vox_size_inv, grid_pts_grad, seed, use_index)


def _inplace_grad(grid_pts_grad):
    if not grid_pts_grad.is_contiguous() or grid_pts_grad.dtype != torch.float32:
        raise RuntimeError("grid_pts_grad must be a contiguous float32 tensor (it is updated in place)")


def _finish(status, what, check_status):
    """Reading the status word waits for the stream, so it is read only on request; a flag
    raised by an earlier unchecked call is reported by the next checked one."""
    if check_status:
        word = int(status.item())
        if word:
            status.zero_()
            raise _lib.SvrError(f"{what}: device status 0x{word:x} (an index out of range was skipped)")


def total_variation(grid_pts, vox_key, weight, vox_size_inv, no_tv_s, tv_sparse, grid_pts_grad, check_status=False,
                    ordered=True):
    """grid_loss_bw.py:13-17 -> tv_compute.cu:23-176.  With tv_sparse, the voxels that take
    part are decided from grid_pts_grad as it is on entry (the reference reads it while it
    adds to it, so its choice depends on thread timing).  ``ordered=True`` visits the voxels
    in the cached spatial order (``voxel_order``); ``False`` in storage order as the
    reference does."""
    assert grid_pts.shape == grid_pts_grad.shape
    assert len(vox_key.shape) == 2 and vox_key.shape[1] == 8
    assert vox_key.shape[0] == vox_size_inv.numel()
    _lib.require_cuda(grid_pts, vox_key, grid_pts_grad)
    _inplace_grad(grid_pts_grad)
    dev = grid_pts.device
    grid = grid_pts.detach().to(torch.float32).contiguous()
    M = grid.shape[0]
    Cn = grid.numel() // max(M, 1)
    key = vox_key.to(torch.int64).contiguous()
    vsi = vox_size_inv.reshape(-1).to(torch.float32).contiguous()
    N = key.shape[0]
    status = _status(dev)
    L = _lib.load()
    valid = torch.empty(max(N * Cn, 1), dtype=torch.uint8, device=dev) if tv_sparse else None
    if ordered and N > 0:
        order, _ = voxel_order(key, M)
        check(L.svr_total_variation_bw_ordered(N, Cn, ptr(order), ptr(key), ptr(grid), M, float(weight), ptr(vsi),
                                               int(bool(no_tv_s)), int(bool(tv_sparse)), ptr(valid),
                                               ptr(grid_pts_grad), ptr(status), stream_ptr(dev)),
              "svr_total_variation_bw_ordered")
    else:
        check(L.svr_total_variation_bw(N, Cn, ptr(key), ptr(grid), M, float(weight), ptr(vsi), int(bool(no_tv_s)),
                                       int(bool(tv_sparse)), ptr(valid), ptr(grid_pts_grad), ptr(status),
                                       stream_ptr(dev)), "svr_total_variation_bw")
    _finish(status, "total_variation", check_status)


def voxel_gradient(grid_pts, vox_key, vox_size_inv, active_list, weight, no_tv_s, tv_sparse, grid_pts_grad,
                   check_status=False, ordered=True):
    """grid_loss_bw.py:19-22 -> vg_compute.cu:23-118 (no_tv_s / tv_sparse unused there too).
    ``ordered`` as in ``total_variation``."""
    assert grid_pts.shape == grid_pts_grad.shape
    assert len(vox_key.shape) == 2 and vox_key.shape[1] == 8
    assert vox_key.shape[0] == vox_size_inv.numel()
    _lib.require_cuda(grid_pts, vox_key, grid_pts_grad)
    _inplace_grad(grid_pts_grad)
    dev = grid_pts.device
    grid = grid_pts.detach().to(torch.float32).contiguous()
    key = vox_key.to(torch.int64).contiguous()
    vsi = vox_size_inv.reshape(-1).to(torch.float32).contiguous()
    act = active_list.to(torch.int32).contiguous()
    N, A = key.shape[0], act.numel()
    status = _status(dev)
    L = _lib.load()
    if ordered and A > 0 and N > 0:
        order, rank = voxel_order(key, grid.numel())
        cnt = torch.empty(N, dtype=torch.int32, device=dev)
        check(L.svr_voxel_gradient_bw_ordered(N, A, ptr(act), ptr(order), ptr(rank), ptr(key), ptr(grid), grid.numel(),
                                              ptr(vsi), float(weight), ptr(cnt), ptr(grid_pts_grad), ptr(status),
                                              stream_ptr(dev)), "svr_voxel_gradient_bw_ordered")
    else:
        check(L.svr_voxel_gradient_bw(N, A, ptr(act), ptr(key), ptr(grid), grid.numel(), ptr(vsi), float(weight),
                                      ptr(grid_pts_grad), ptr(status), stream_ptr(dev)), "svr_voxel_gradient_bw")
    _finish(status, "voxel_gradient", check_status)


def points_loss(points_in_grid, grid_pts, vox_key, grid_voxel_coord, grid_voxel_size, grid_res, grid_mask,
                grid_keys, grid2voxel, weight, vox_size_inv, no_tv_s, tv_sparse, grid_pts_grad, use_index=True,
                check_status=False):
    """grid_loss_bw.py:34-37 -> pl_compute.cu:14-108 (vox_size_inv, no_tv_s, tv_sparse unused
    there too)."""
    assert grid_pts.shape == grid_pts_grad.shape
    assert len(vox_key.shape) == 2 and vox_key.shape[1] == 8
    _lib.require_cuda(points_in_grid, grid_pts, vox_key, grid_keys, grid_pts_grad)
    _inplace_grad(grid_pts_grad)
    dev = grid_pts.device
    pts = points_in_grid.to(torch.float32).contiguous()
    keys = grid_keys.to(torch.int32).contiguous()
    g2v = grid2voxel.to(torch.int32).contiguous()
    coords = grid_voxel_coord.to(torch.float32).contiguous()
    sizes = grid_voxel_size.reshape(-1).to(torch.float32).contiguous()
    key = vox_key.to(torch.int64).contiguous()
    grid = grid_pts.detach().to(torch.float32).contiguous()
    mask = grid_mask.contiguous()
    didx = dense_index(grid_keys, grid_res) if use_index else None
    status = _status(dev)
    check(_lib.load().svr_points_loss_bw(pts.shape[0], ptr(pts), keys.numel(), ptr(keys), ptr(g2v), int(grid_res),
                                         ptr(mask), ptr(didx), ptr(coords), ptr(sizes), key.shape[0], ptr(key),
                                         ptr(grid), grid.numel(), float(weight), ptr(grid_pts_grad), ptr(status),
                                         stream_ptr(dev)), "svr_points_loss_bw")
    _finish(status, "points_loss", check_status)
