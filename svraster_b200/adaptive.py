"""Adaptive pruning / subdivision and training statistics on the GPU.

Interfaces of the reference's src/utils/octree_utils.py (gen_children, octpath_decoding,
build_grid_pts_link) and src/sparse_voxel_gears/adaptive.py (compute_training_stat, pruning,
subdividing, mask_cat_perm, agg_voxel_into_grid_pts, subdivide_by_interp): same names,
argument meaning and results.  The grid-point link (a unique over the 8N corner coordinates),
the trilinear child values, the mean aggregation into grid points and the per-voxel statistics
run as this library's kernels (csrc/adaptive.cu); the statistics come from one batched forward
over all views instead of one render per camera.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_ptr
from . import utils
from .meta import MAX_NUM_LEVELS


# ----------------------------------------------------------------------------- octree helpers
def level_2_vox_size(scene_extent, octlevel):
    """scene_extent * 2^-level (octree_utils.py:51-59)."""
    return torch.ldexp(scene_extent.expand(octlevel.shape).contiguous(), -octlevel)


def octpath_decoding(octpath, octlevel, scene_center, scene_extent):
    """Voxel centres [N,3] and sizes [N,1] (octree_utils.py:99-125)."""
    octpath = octpath.reshape(-1, 1)
    octlevel = octlevel.reshape(-1, 1)
    vox_size = level_2_vox_size(scene_extent, octlevel)
    ijk = utils.octpath_2_ijk(octpath, octlevel)
    return (scene_center - 0.5 * scene_extent) + (ijk + 0.5) * vox_size, vox_size


def gen_children(octpath, octlevel):
    """The eight children (octpath, octlevel) of each voxel, children of a voxel consecutive in
    octant order (octree_utils.py:162-198)."""
    octpath = octpath.reshape(-1, 1)
    octlevel = octlevel.reshape(-1, 1) + 1
    if int(octlevel.max()) > MAX_NUM_LEVELS:
        raise ValueError("maximum level out of bound after subdivision")
    octant = torch.arange(8, dtype=torch.int64, device=octpath.device)
    shift = 3 * (MAX_NUM_LEVELS - octlevel.to(torch.int64))
    children = (octpath | (octant.view(1, 8) << shift)).reshape(-1, 1)
    return children, octlevel.repeat_interleave(8, dim=0)


def build_grid_pts_link(octpath, octlevel):
    """Corner grid points shared between voxels (octree_utils.py:203-222):
    grid_pts_key int64 [M,3] (finest-level coordinates, lexicographic order) and
    vox_key int64 [N,8] (indices of each voxel's corners)."""
    L = _lib.load()
    dev = octpath.device
    _lib.require_cuda(octpath)
    octpath = octpath.reshape(-1).to(torch.int64).contiguous()
    octlevel = octlevel.reshape(-1).to(torch.int8).contiguous()
    N = octpath.numel()
    keys = torch.empty(max(8 * N, 1), 3, dtype=torch.int64, device=dev)
    vox_key = torch.empty(N, 8, dtype=torch.int64, device=dev)
    wsb = L.svr_grid_link_workspace_bytes(N)
    ws = torch.empty(max(int(wsb), 16), dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    M = C.c_int64(0)
    check(L.svr_grid_link(N, ptr(octpath), ptr(octlevel), ptr(ws), wsb, ptr(keys), ptr(vox_key), C.byref(M),
                          ptr(status), stream_ptr(dev)), "svr_grid_link")
    if int(status.item()):
        raise RuntimeError("build_grid_pts_link: octree level out of range")
    return keys[: M.value].contiguous(), vox_key


def compute_gridpoints_xyz(gridpts, scene_center, scene_extent):
    """World positions of finest-level grid coordinates (octree_utils.py:146-160)."""
    finest = level_2_vox_size(scene_extent, torch.tensor(MAX_NUM_LEVELS, dtype=torch.int64,
                                                         device=gridpts.device))
    return (scene_center - 0.5 * scene_extent) + gridpts * finest


# ----------------------------------------------------------------------------- per-voxel data
def mask_cat_perm(tensor, kept_idx=None, cat_tensor=None, perm=None):
    """Select kept rows, append cat_tensor, permute (adaptive.py:330-347)."""
    if kept_idx is None and cat_tensor is None and perm is None:
        raise ValueError("mask_cat_perm: nothing to do")
    dev = tensor.device
    if kept_idx is not None:
        tensor = tensor[kept_idx.to(dev)]
    if cat_tensor is not None:
        tensor = torch.cat([tensor, cat_tensor.to(dev)])
    if perm is not None:
        if len(perm) != len(tensor):
            raise ValueError("mask_cat_perm: permutation length")
        tensor = tensor[perm.to(dev)]
    return tensor.contiguous()


def agg_voxel_into_grid_pts(num_grid_pts, vox_key, vox_val, reduce="mean"):
    """Mean of the corner values of all voxels sharing each grid point (adaptive.py:349-372,
    index_reduce_ mean with include_self=False into zeros).  vox_val [N,8,*] -> [M,*]."""
    if reduce != "mean":
        raise NotImplementedError("agg_voxel_into_grid_pts: only reduce='mean'")
    L = _lib.load()
    dev = vox_val.device
    _lib.require_cuda(vox_val)
    ch = tuple(vox_val.shape[2:])
    Cn = int(np.prod(ch)) if ch else 1
    val = vox_val.reshape(vox_val.shape[0], 8, Cn).to(torch.float32).contiguous()
    key = vox_key.to(dev).reshape(-1, 8).to(torch.int64).contiguous()
    M = int(num_grid_pts)
    out = torch.empty(M, Cn, dtype=torch.float32, device=dev)
    cnt = torch.empty(max(M, 1), dtype=torch.float32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    check(L.svr_agg_voxel_into_grid_pts(val.shape[0], Cn, ptr(key), ptr(val), M, ptr(out), ptr(cnt), ptr(status),
                                        stream_ptr(dev)), "svr_agg_voxel_into_grid_pts")
    if int(status.item()):
        raise RuntimeError("agg_voxel_into_grid_pts: vox_key out of range")
    return out.reshape(M, *ch).contiguous()


def subdivide_by_interp(vox_val):
    """Corner values of the eight children by trilinear interpolation of the parent's
    (adaptive.py:374-411).  vox_val [N,8,*] -> [8N,8,*], children in gen_children order."""
    L = _lib.load()
    dev = vox_val.device
    _lib.require_cuda(vox_val)
    ch = tuple(vox_val.shape[2:])
    Cn = int(np.prod(ch)) if ch else 1
    val = vox_val.reshape(vox_val.shape[0], 8, Cn).to(torch.float32).contiguous()
    out = torch.empty(8 * val.shape[0], 8, Cn, dtype=torch.float32, device=dev)
    check(L.svr_subdivide_interp(val.shape[0], Cn, ptr(val), ptr(out), stream_ptr(dev)), "svr_subdivide_interp")
    return out.reshape(8 * val.shape[0], 8, *ch).contiguous()


# ----------------------------------------------------------------------------- statistics
def _view_dict(cam, device):
    """Camera (svraster_b200.synthetic.Camera or the reference's Camera) as a render view."""
    t = lambda a: torch.as_tensor(np.asarray(a.detach().cpu() if torch.is_tensor(a) else a),
                                  dtype=torch.float32).to(device).contiguous()
    W = getattr(cam, "width", None) or cam.image_width
    H = getattr(cam, "height", None) or cam.image_height
    return dict(width=int(W), height=int(H), tanfovx=float(cam.tanfovx), tanfovy=float(cam.tanfovy),
                cx=float(cam.cx), cy=float(cam.cy), near=float(getattr(cam, "near", 0.02)), w2c=t(cam.w2c),
                c2w=t(cam.c2w), bg=torch.zeros(3, device=device))


def compute_training_stat(camera_lst, octpath, vox_center, vox_size, is_leaf, geos, s_val, n_samp=3):
    """Per-voxel max blending weight, minimum sampling interval and visible-view count over the
    cameras (adaptive.py:80-113), from one batched forward with per-view max-weight tracking.
    geos f32[N,8] are the corner SDF values, s_val the NeuS sharpness (tensor [1])."""
    from .raster import RasterState
    L = _lib.load()
    dev = vox_center.device
    _lib.require_cuda(vox_center)
    N = vox_center.shape[0]
    views = [_view_dict(c, dev) for c in camera_lst]
    V = len(views)
    centers = vox_center.reshape(N, 3).to(torch.float32).contiguous()
    lengths = vox_size.reshape(N).to(torch.float32).contiguous()
    leaf = is_leaf.reshape(N).to(torch.uint8).contiguous()
    paths = octpath.reshape(N).to(torch.int64).contiguous()
    geos_c = geos.reshape(N, 8).to(torch.float32).contiguous()
    s = s_val.reshape(1).to(torch.float32).contiguous()
    rgbs = torch.zeros(N, 3, device=dev)          # colour does not enter the weights
    max_w = torch.zeros(N, 1, device=dev)
    min_samp = torch.full((N, 1), 1e30, device=dev)
    view_cnt = torch.zeros(N, 1, device=dev)
    step = 64                                     # views per batch (SVR_MAX_VIEWS is 128)
    for v0 in range(0, V, step):
        part = views[v0:v0 + step]
        st = RasterState(part, N, dev)
        st.preprocess(paths, centers, lengths, leaf)
        st.bin(paths)
        P = st.total_pix
        color = torch.empty(3 * P, device=dev)
        T = torch.empty(P, device=dev)
        depth = torch.empty(4 * P, device=dev)
        normal = torch.empty(3 * P, device=dev)
        mw = torch.zeros(len(part), N, device=dev)
        check(L.svr_render_fwd_max_w_views(st.views, st.n_views, N, st.num_rendered, int(n_samp), 1, 1, ptr(centers),
                                           ptr(lengths), ptr(geos_c), ptr(rgbs), 1, ptr(s), ptr(st.geom),
                                           ptr(st.binning), ptr(st.image), ptr(color), ptr(depth), ptr(normal), ptr(T),
                                           ptr(mw), stream_ptr(dev)), "svr_render_fwd_max_w_views")
        pos = torch.stack([d["c2w"][:3, 3] for d in part]).contiguous()
        look = torch.stack([d["c2w"][:3, 2] for d in part]).contiguous()
        pix = torch.tensor([np.float32(2 * d["tanfovx"] / d["width"]) for d in part], device=dev)
        check(L.svr_training_stat_reduce(len(part), N, ptr(mw), ptr(centers), ptr(pos), ptr(look), ptr(pix),
                                         ptr(max_w), ptr(min_samp), ptr(view_cnt), stream_ptr(dev)),
              "svr_training_stat_reduce")
    return {"max_w": max_w, "min_samp_interval": min_samp, "view_cnt": view_cnt}


# ----------------------------------------------------------------------------- model mixin
class SVAdaptive:
    """Pruning and subdivision of a sparse-voxel model that keeps the reference's layout:
    per_voxel_attr_lst (octpath, octlevel, vox_center, vox_size, is_leaf, ...),
    per_voxel_param_lst and grid_pts_param_lst attribute names, vox_key / grid_pts_key,
    scene_center, scene_extent, outside_level (adaptive.py:29-72, 143-327).  Optimizer states
    of the reshaped parameters are dropped and recreated empty, as there."""

    @torch.no_grad()
    def pruning(self, prune_mask):
        kept_idx = (~prune_mask.reshape(-1)).nonzero().reshape(-1)
        self._drop_optimizer_states()
        for name in self.per_voxel_attr_lst:
            setattr(self, name, mask_cat_perm(getattr(self, name), kept_idx=kept_idx))
        for name in self.per_voxel_param_lst:
            setattr(self, name, mask_cat_perm(getattr(self, name).detach(), kept_idx=kept_idx).requires_grad_())
        self._relink_grid_pts(kept_idx, None)
        self._renew_optimizer_states()

    @torch.no_grad()
    def subdividing(self, subdivide_mask):
        sub = subdivide_mask.reshape(-1)
        depth_rel = self.octlevel.reshape(-1) - self.outside_level
        keep_parent = sub & (depth_rel >= 9)          # deep parents stay as non-leaf voxels
        kept_idx = ((~sub) | keep_parent).nonzero().reshape(-1)
        sub_idx = sub.nonzero().reshape(-1)
        parent_idx = keep_parent.nonzero().reshape(-1)
        self._drop_optimizer_states()
        octpath, octlevel = gen_children(self.octpath[sub_idx], self.octlevel[sub_idx])
        vox_center, vox_size = octpath_decoding(octpath, octlevel, self.scene_center, self.scene_extent)
        children = {"octpath": octpath, "octlevel": octlevel, "vox_center": vox_center, "vox_size": vox_size}
        for name in self.per_voxel_attr_lst:
            cur = getattr(self, name)
            if name in children:
                add = children[name]
            elif name == "is_leaf":
                cur[parent_idx] = False
                add = torch.ones_like(cur[sub_idx]).repeat_interleave(8, dim=0)
            else:
                add = cur[sub_idx].repeat_interleave(8, dim=0)
            setattr(self, name, mask_cat_perm(cur, kept_idx=kept_idx, cat_tensor=add))
        for name in self.per_voxel_param_lst:
            cur = getattr(self, name).detach()
            setattr(self, name, mask_cat_perm(cur, kept_idx=kept_idx,
                                              cat_tensor=cur[sub_idx].repeat_interleave(8, dim=0)).requires_grad_())
        self._relink_grid_pts(kept_idx, sub_idx)
        self._renew_optimizer_states()

    def _relink_grid_pts(self, kept_idx, sub_idx):
        old_vox_key = self.vox_key
        self.grid_pts_key, self.vox_key = build_grid_pts_link(self.octpath, self.octlevel)
        M = len(self.grid_pts_key)
        for name in self.grid_pts_param_lst:
            per_vox = getattr(self, name).detach()[old_vox_key]
            add = subdivide_by_interp(per_vox[sub_idx]) if sub_idx is not None else None
            new_vox = mask_cat_perm(per_vox, kept_idx=kept_idx, cat_tensor=add)
            setattr(self, name, agg_voxel_into_grid_pts(M, self.vox_key, new_vox).requires_grad_())

    def _drop_optimizer_states(self):
        opt = getattr(self, "optimizer", None)
        if opt is None:
            return
        for name in self.per_voxel_param_lst + self.grid_pts_param_lst:
            opt.state.pop(getattr(self, name), None)

    def _renew_optimizer_states(self):
        opt = getattr(self, "optimizer", None)
        if opt is None:
            return
        groups = {g.get("name"): g for g in opt.param_groups}
        for name in self.per_voxel_param_lst + self.grid_pts_param_lst:
            g = groups.get(name)
            if g is None:
                continue
            g["params"][0] = getattr(self, name)
            opt.state[g["params"][0]] = {}
