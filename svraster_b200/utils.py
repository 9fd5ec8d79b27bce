"""Drop-in replacement of ``svraster_cuda.utils`` (cuda/svraster_cuda/utils.py).

``valid_gradient_table`` runs on the sm_100a library.  The camera / octree helpers
(``is_in_cone``, ``compute_rd``, ``depth2pts``, ``voxel_order_rank``, ``ijk_2_octpath``,
``octpath_2_ijk``) are initialisation / evaluation utilities outside the rasterizer hot
path; they are restated as device tensor expressions with the same semantics
(cuda/src/utils.cu:23-189).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check, ptr, stream_ptr
from .meta import MAX_NUM_LEVELS


def _rep3(q):
    v = 0
    for _ in range(MAX_NUM_LEVELS):
        v = (v << 3) | q
    return v


def voxel_order_rank(octree_paths):
    """utils.cu:104-127 -> int64 [8, P]: octree path XOR the octant pattern."""
    p = octree_paths.reshape(-1).to(torch.int64)
    return torch.stack([p ^ _rep3(q) for q in range(8)], 0)


def is_in_cone(pts, cam):
    """utils.cu:23-45."""
    assert torch.is_tensor(pts)
    assert pts.device == cam.w2c.device
    assert len(pts.shape) == 2 and pts.shape[1] == 3
    w2c = cam.w2c.to(torch.float32)
    pc = pts @ w2c[:3, :3].T + w2c[:3, 3]
    return (pc[:, 2] > cam.near) & (pc[:, 0].abs() <= cam.tanfovx * pc[:, 2]) & \
        (pc[:, 1].abs() <= cam.tanfovy * pc[:, 2])


def _cam_dirs(width, height, cx, cy, tanfovx, tanfovy, c2w):
    dev = c2w.device
    y, x = torch.meshgrid(torch.arange(height, device=dev, dtype=torch.float32),
                          torch.arange(width, device=dev, dtype=torch.float32), indexing="ij")
    cam = torch.stack([(x + 0.5 - cx) * 2.0 * tanfovx / float(width),
                       (y + 0.5 - cy) * 2.0 * tanfovy / float(height), torch.ones_like(x)], 0)
    return torch.einsum("ij,jhw->ihw", c2w[:3, :3].to(torch.float32), cam)


def compute_rd(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix):
    """utils.cu:47-72 -> [3, H, W] unnormalised world ray directions."""
    assert torch.is_tensor(c2w_matrix)
    return _cam_dirs(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix)


def depth2pts(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix, depth):
    """utils.cu:74-102 -> [3, H, W]."""
    assert torch.is_tensor(c2w_matrix)
    assert depth.device == c2w_matrix.device
    assert depth.numel() == width * height
    d = _cam_dirs(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix)
    return c2w_matrix[:3, 3].to(torch.float32).view(3, 1, 1) + depth.reshape(1, height, width) * d


def ijk_2_octpath(ijk, octlevel):
    """utils.cu:129-158."""
    assert torch.is_tensor(ijk) and torch.is_tensor(octlevel)
    assert len(ijk.shape) == 2 and ijk.shape[1] == 3
    assert ijk.numel() == octlevel.numel() * 3
    assert ijk.dtype == torch.int64
    assert octlevel.dtype == torch.int8
    lv = octlevel.reshape(-1).to(torch.int64)
    path = torch.zeros(len(lv), dtype=torch.int64, device=ijk.device)
    i, j, k = ijk[:, 0], ijk[:, 1], ijk[:, 2]
    for l in range(MAX_NUM_LEVELS):
        bits = (((i >> l) & 1) << 2) | (((j >> l) & 1) << 1) | ((k >> l) & 1)
        path |= bits << (3 * l)
    return (path << (3 * (MAX_NUM_LEVELS - lv))).reshape(-1, 1)


def octpath_2_ijk(octpath, octlevel):
    """utils.cu:160-189."""
    assert torch.is_tensor(octpath) and torch.is_tensor(octlevel)
    assert octpath.numel() == octlevel.numel()
    assert octpath.dtype == torch.int64
    assert octlevel.dtype == torch.int8
    lv = octlevel.reshape(-1).to(torch.int64)
    p = octpath.reshape(-1) >> (3 * (MAX_NUM_LEVELS - lv))
    ijk = torch.zeros(len(lv), 3, dtype=torch.int64, device=octpath.device)
    for l in range(MAX_NUM_LEVELS):
        b = p & 7
        ijk[:, 0] |= ((b >> 2) & 1) << l
        ijk[:, 1] |= ((b >> 1) & 1) << l
        ijk[:, 2] |= (b & 1) << l
        p = p >> 3
    return ijk


def valid_gradient_table(vox_center, vox_size, scene_center, inside_extent, grid_res, is_leaf):
    """cuda/svraster_cuda/utils.py:133-171 -> (grid_mask bool[res^3], grid_keys int32[G],
    grid2voxel int32[G]) with keys already sorted (src/utils/octree_utils.py:303-308 sorts
    them again, which is then the identity)."""
    _lib.require_cuda(vox_center, vox_size)
    L = _lib.load()
    dev = vox_center.device
    centers = vox_center.to(torch.float32).contiguous()
    sizes = vox_size.reshape(-1).to(torch.float32).contiguous()
    sc = torch.as_tensor(scene_center, dtype=torch.float32, device=dev).reshape(-1).contiguous()
    leaf = is_leaf.reshape(-1).to(torch.uint8).contiguous()
    N = centers.shape[0]
    res = 1 << int(grid_res)
    st = stream_ptr(dev)
    ws = torch.empty(max(L.svr_valid_table_workspace_bytes(N, 0), 16), dtype=torch.uint8, device=dev)
    cnt = C.c_int64(0)
    check(L.svr_valid_table_count(N, ptr(centers), ptr(sizes), ptr(sc), float(inside_extent), int(grid_res),
                                  ptr(leaf), ptr(ws), C.byref(cnt), st), "svr_valid_table_count")
    G = int(cnt.value)
    need = L.svr_valid_table_workspace_bytes(N, G)
    if need > ws.numel():
        ws2 = torch.empty(need, dtype=torch.uint8, device=dev)
        ws2[: ws.numel()].copy_(ws)
        ws = ws2
    grid_mask = torch.empty(res ** 3, dtype=torch.bool, device=dev)
    keys = torch.empty(max(G, 1), dtype=torch.int32, device=dev)
    g2v = torch.empty(max(G, 1), dtype=torch.int32, device=dev)
    check(L.svr_valid_table_fill(N, ptr(centers), ptr(sizes), ptr(sc), float(inside_extent), int(grid_res),
                                 ptr(leaf), G, ptr(ws), ptr(grid_mask), ptr(keys), ptr(g2v), st),
          "svr_valid_table_fill")
    return grid_mask, keys[:G], g2v[:G]
