"""Drop-in replacement of ``svraster_cuda.grid_loss_bw`` (cuda/svraster_cuda/grid_loss_bw.py).

The functions accumulate into ``grid_pts_grad`` in place and return ``None``, as the
reference's do.  ``laplacian_smoothness`` and ``grid_eikonal`` run on the sm_100a library.
The reference seeds their jitter with the GPU clock (ls_compute.cu:43, ge_compute.cu:74);
here the seed comes from torch's host RNG unless ``seed=`` is given, so runs are
reproducible under ``torch.manual_seed``.
"""
from __future__ import annotations

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


def total_variation(grid_pts, vox_key, weight, vox_size_inv, no_tv_s, tv_sparse, grid_pts_grad):
    """grid_loss_bw.py:13-17 (off under the shipped SDF settings, train.py:1355)."""
    raise NotImplementedError("total_variation is not part of the shipped SDF path")


def voxel_gradient(grid_pts, vox_key, vox_size_inv, active_list, weight, no_tv_s, tv_sparse, grid_pts_grad):
    """grid_loss_bw.py:19-22."""
    raise NotImplementedError("voxel_gradient is not implemented in this build")


def points_loss(points_in_grid, grid_pts, vox_key, grid_voxel_coord, grid_voxel_size, grid_res, grid_mask,
                grid_keys, grid2voxel, weight, vox_size_inv, no_tv_s, tv_sparse, grid_pts_grad):
    """grid_loss_bw.py:34-37 (off by default, src/config.py:170)."""
    raise NotImplementedError("points_loss is not part of the shipped SDF path")
