"""TSDF fusion on the sm_100a library: drop-in for ``Fuser`` of src/utils/fuser_utils.py:18-156.

``Fuser(xyz, bandwidth, ...)`` keeps the reference's constructor arguments and the
``integrate(cam, depth, alpha=None)`` / ``tsdf`` interface; ``integrate_batch`` folds many
views in one launch.  ``precision="fp64"`` keeps the weighted running sums in float64 (the
reference accumulates in float32, which stays the default).  Feature fusion
(``feat_dim > 0``), normal weighting and half-precision storage are outside the SDF
extraction path and raise ``NotImplementedError``.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_ptr


def _cam_view(cam):
    """svr_view_t fields + the double-precision projection constants of a camera object
    with the reference Camera interface (w2c / c2w tensors, tanfovx, tanfovy, cx_p, cy_p,
    image_width, image_height)."""
    W, H = int(cam.image_width), int(cam.image_height)
    cx_p = float(getattr(cam, "cx_p", 0.5))
    cy_p = float(getattr(cam, "cy_p", 0.5))
    view = dict(width=W, height=H, tanfovx=float(cam.tanfovx), tanfovy=float(cam.tanfovy), cx=cx_p * W,
                cy=cy_p * H, near=float(getattr(cam, "near", 0.02)),
                w2c=cam.w2c.detach().to(torch.float32).contiguous(),
                c2w=cam.c2w.detach().to(torch.float32).contiguous(), bg=None)
    proj = [float(cam.tanfovx), float(cam.tanfovy), cx_p, cy_p]
    return view, proj


class Fuser:
    def __init__(self, xyz, bandwidth, use_trunc=True, fuse_tsdf=True, feat_dim=0, alpha_thres=0.5,
                 crop_border=0.0, normal_weight=False, depth_weight=False, border_weight=False,
                 max_norm_dist=10., use_half=False, precision="fp32"):
        assert len(xyz.shape) == 2
        assert xyz.shape[1] == 3
        if feat_dim > 0:
            raise NotImplementedError("feature fusion is not part of the SDF extraction path")
        if normal_weight:
            raise NotImplementedError("normal weighting is not part of the SDF extraction path")
        if use_half:
            raise NotImplementedError("half-precision accumulators are not supported")
        if not fuse_tsdf:
            raise NotImplementedError("weight-only fusion is not part of the SDF extraction path")
        _lib.require_cuda(xyz)
        self.xyz = xyz.detach().to(torch.float32).contiguous()
        self.bandwidth = bandwidth
        self.use_trunc = use_trunc
        self.fuse_tsdf = fuse_tsdf
        self.feat_dim = feat_dim
        self.alpha_thres = alpha_thres
        self.crop_border = crop_border
        self.depth_weight = depth_weight
        self.border_weight = border_weight
        self.max_norm_dist = max_norm_dist
        self.fp64 = precision == "fp64"
        dt = torch.float64 if self.fp64 else torch.float32
        self.weight = torch.zeros([len(xyz), 1], dtype=dt, device=xyz.device)
        self.sd_val = torch.zeros([len(xyz), 1], dtype=dt, device=xyz.device)
        self.feat = torch.zeros([len(xyz), 0], dtype=dt, device=xyz.device)
        if torch.is_tensor(bandwidth):
            self._inv_trunc = (1 / bandwidth.reshape(-1).to(torch.float32)).contiguous()
            self._trunc = 1.0
        else:
            self._inv_trunc = None
            self._trunc = float(bandwidth)

    def integrate_batch(self, cams, depths, alphas=None):
        """Integrate several views in one launch; depths / alphas are [1,H,W] (or [H,W]) maps."""
        if len(cams) == 0:
            return
        for i in range(0, len(cams), _lib.SVR_MAX_VIEWS):
            self._integrate(cams[i:i + _lib.SVR_MAX_VIEWS], depths[i:i + _lib.SVR_MAX_VIEWS],
                            None if alphas is None else alphas[i:i + _lib.SVR_MAX_VIEWS])

    def integrate(self, cam, depth, feat=None, alpha=None):
        """fuser_utils.py:54-148 for one view."""
        if feat is not None:
            raise NotImplementedError("feature fusion is not part of the SDF extraction path")
        self._integrate([cam], [depth], None if alpha is None else [alpha])

    def _integrate(self, cams, depths, alphas):
        dev = self.xyz.device
        views, proj = [], []
        for c in cams:
            v, p = _cam_view(c)
            v["bg"] = torch.zeros(3, device=dev)
            views.append(v)
            proj += p
        arr, _, _ = _lib.make_views(views)
        depth = torch.cat([d.detach().reshape(-1).to(torch.float32) for d in depths]).contiguous()
        alpha = None
        if alphas is not None:
            alpha = torch.cat([a.detach().reshape(-1).to(torch.float32) for a in alphas]).contiguous()
        proj_h = (len(proj) * _lib.C.c_double)(*proj)
        check(_lib.load().svr_tsdf_integrate(arr, proj_h, len(views), self.xyz.shape[0], ptr(self.xyz), ptr(depth), 1,
                                             0, ptr(alpha), 1, 0, 0, ptr(self._inv_trunc), self._trunc,
                                             float(self.crop_border), float(self.alpha_thres), int(self.use_trunc),
                                             int(self.depth_weight), int(self.border_weight),
                                             float(self.max_norm_dist), int(self.fp64), ptr(self.weight),
                                             ptr(self.sd_val), stream_ptr(dev)), "svr_tsdf_integrate")
        self._keep = (views, depth, alpha)

    @property
    def feature(self):
        return self.feat / self.weight

    @property
    def tsdf(self):
        return self.sd_val / self.weight
