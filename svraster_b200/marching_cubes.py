"""Drop-in replacement of ``svraster_cuda.marching_cubes`` (cuda/svraster_cuda/marching_cubes.py)
on the sm_100a library.

``torch_marching_cubes_grid`` returns the same vertices (lexicographically sorted unique
rows) and faces as the reference: the vertex interpolation uses the reference's
separately-rounded float32 operations, so vertices and topology are bit-identical given the
same SDF values.  ``chunk_sz`` is accepted for compatibility; the result does not depend on
it (the reference's per-chunk results are merged by a global unique), so all voxels are
processed in one pass.  ``fp64=True`` interpolates in double precision instead.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check, ptr, stream_ptr


def torch_marching_cubes_grid(grid_pts_val, grid_pts_xyz, vox_key, iso, chunk_sz=10_000_000, fp64=False):
    """marching_cubes.py:278-312."""
    _lib.require_cuda(grid_pts_val, grid_pts_xyz, vox_key)
    dev = grid_pts_val.device
    val = grid_pts_val.detach().reshape(-1).to(torch.float32).contiguous()
    xyz = grid_pts_xyz.detach().to(torch.float32).contiguous()
    key = vox_key.to(torch.int64).contiguous()
    n_vox = key.shape[0]
    L = _lib.load()
    st = stream_ptr(dev)
    ws = torch.empty(max(L.svr_mc_workspace_bytes(n_vox, 0), 16), dtype=torch.uint8, device=dev)
    ntri = C.c_int64(0)
    check(L.svr_mc_count(n_vox, ptr(key), val.numel(), ptr(val), float(iso), ptr(ws), C.byref(ntri), st),
          "svr_mc_count")
    T = int(ntri.value)
    if T == 0:
        return (torch.zeros(0, 3, dtype=torch.float32, device=dev), torch.zeros(0, 3, dtype=torch.int64, device=dev))
    need = L.svr_mc_workspace_bytes(n_vox, T)
    if need > ws.numel():
        ws2 = torch.empty(need, dtype=torch.uint8, device=dev)
        ws2[: ws.numel()].copy_(ws)
        ws = ws2
    verts = torch.empty(3 * T, 3, dtype=torch.float32, device=dev)
    faces = torch.empty(T, 3, dtype=torch.int64, device=dev)
    nv = C.c_int64(0)
    check(L.svr_mc_emit(n_vox, ptr(key), ptr(val), ptr(xyz), float(iso), T, int(fp64), ptr(ws), ptr(verts),
                        ptr(faces), C.byref(nv), st), "svr_mc_emit")
    return verts[: int(nv.value)], faces


def torch_marching_cubes_voxels(unit_val, unit_xyz, iso):
    """marching_cubes.py:315-380: the same on per-voxel corner values [n,8] / positions [n,8,3]."""
    n = unit_val.shape[0]
    key = torch.arange(n * 8, dtype=torch.int64, device=unit_val.device).view(n, 8)
    return torch_marching_cubes_grid(unit_val.reshape(-1), unit_xyz.reshape(-1, 3), key, iso)
