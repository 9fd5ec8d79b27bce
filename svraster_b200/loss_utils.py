"""Drop-in for the normal-from-depth consistency losses of src/utils/loss_utils.py.

``NormalDepthConsistencyLoss`` (loss_utils.py:345-379) and ``NormalMedianConsistencyLoss``
(loss_utils.py:381-407) keep the reference's constructor arguments, ``is_active`` and
``__call__(cam, render_pkg, iteration)``; the loss is a torch scalar that back-propagates into
``render_pkg['raw_depth']`` and ``render_pkg['raw_normal']`` as the reference's does.  The
loss and both gradients come from one sm_100a launch (``svr_normal_depth_loss``); the
backward only scales the stored gradients.  ``normal_depth_loss_views`` is the batched form
for packed multi-view planes (the training step's upstream gradient planes).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_ptr


def _cam_desc(cam, dev):
    """A view dict for a reference camera (image_width, image_height, c2w tensor) or one of
    ``svraster_b200.synthetic``'s (width, height, c2w array)."""
    W = int(getattr(cam, "image_width", getattr(cam, "width", 0)))
    H = int(getattr(cam, "image_height", getattr(cam, "height", 0)))
    c2w = cam.c2w
    c2w = (c2w.detach() if torch.is_tensor(c2w) else torch.as_tensor(np.asarray(c2w)))
    c2w = c2w.to(dev, torch.float32).contiguous()
    return dict(width=W, height=H, tanfovx=float(cam.tanfovx), tanfovy=float(cam.tanfovy), cx=float(cam.cx),
                cy=float(cam.cy), w2c=c2w, c2w=c2w, bg=c2w)


def normal_depth_loss_views(cams, depth, normal, T, mode, ks=3, tol_cos=-1.0, weight=1.0, grad_depth=None,
                            grad_normal=None, loss_out=None):
    """Per-view losses f64[n_views] (times ``weight``) for packed planes (depth f32[4*P],
    normal f32[3*P], T f32[P], P the views' total pixels).  ``cams`` holds cameras or view
    dicts of ``_lib.make_views`` (with device c2w tensors, as a render batch keeps them;
    they skip the per-call upload of the camera matrices).  The gradients are ADDED into
    ``grad_depth`` / ``grad_normal`` (allocated as zeros when not given).  mode "dmean" or
    "dmed".  Returns (loss, grad_depth, grad_normal)."""
    dev = depth.device
    _lib.require_cuda(depth, normal, T)
    descs = [c if isinstance(c, dict) else _cam_desc(c, dev) for c in cams]
    views, _, total = _lib.make_views(descs)
    depth = depth.detach().to(torch.float32).contiguous()
    normal = normal.detach().to(torch.float32).contiguous()
    if depth.numel() != 4 * total or normal.numel() != 3 * total:
        raise ValueError("normal_depth_loss_views: planes do not match the views' pixel count")
    if grad_depth is None:
        grad_depth = torch.zeros_like(depth)
    if grad_normal is None:
        grad_normal = torch.zeros_like(normal)
    if loss_out is None:
        loss_out = torch.zeros(len(cams), dtype=torch.float64, device=dev)
    Tc = None
    if mode == "dmean":
        Tc = T.detach().to(torch.float32).contiguous()
        if Tc.numel() != total:
            raise ValueError("normal_depth_loss_views: T does not match the views' pixel count")
    elif mode != "dmed":
        raise ValueError("mode must be 'dmean' or 'dmed'")
    check(_lib.load().svr_normal_depth_loss(views, len(cams), 0 if mode == "dmean" else 1, int(ks), float(tol_cos),
                                            float(weight), ptr(depth), ptr(normal), ptr(Tc), ptr(loss_out),
                                            ptr(grad_depth), ptr(grad_normal), stream_ptr(dev)),
          "svr_normal_depth_loss")
    return loss_out, grad_depth, grad_normal


class _NormalLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, depth, normal, T, cam, mode, ks, tol_cos):
        loss, gd, gn = normal_depth_loss_views([cam], depth, normal, T, mode, ks, tol_cos)
        ctx.save_for_backward(gd, gn)
        return loss[0].to(torch.float32)

    @staticmethod
    def backward(ctx, g):
        gd, gn = ctx.saved_tensors
        return gd * g, gn * g, None, None, None, None, None


class NormalDepthConsistencyLoss:
    """loss_utils.py:345-379: rendered normal against the alpha-weighted negated normal of the
    mean-depth surface (depth2normal with ``ks`` and the tolerance ``tol_deg``)."""

    def __init__(self, iter_from, iter_end, ks, tol_deg):
        self.iter_from = iter_from
        self.iter_end = iter_end
        self.ks = ks
        self.tol_cos = np.cos(np.deg2rad(tol_deg))

    def is_active(self, iteration):
        return iteration >= self.iter_from and iteration <= self.iter_end

    def __call__(self, cam, render_pkg, iteration):
        assert "raw_T" in render_pkg, "Forgot to set `output_T=True` when calling render?"
        assert "raw_depth" in render_pkg, "Forgot to set `output_depth=True` when calling render?"
        assert "raw_normal" in render_pkg, "Forgot to set `output_normal=True` when calling render?"
        if not self.is_active(iteration):
            return 0
        # the comparison happens in float32, as the reference's tensor comparison does
        tol = float(np.float32(self.tol_cos)) if self.tol_cos > 0 else -1.0
        return _NormalLoss.apply(render_pkg["raw_depth"], render_pkg["raw_normal"], render_pkg["raw_T"].detach(),
                                 cam, "dmean", int(self.ks), tol)


class NormalMedianConsistencyLoss:
    """loss_utils.py:381-407: rendered normal against the negated normal of the median-depth
    surface (ks 3, no tolerance)."""

    def __init__(self, iter_from, iter_end):
        self.iter_from = iter_from
        self.iter_end = iter_end

    def is_active(self, iteration):
        return iteration >= self.iter_from and iteration <= self.iter_end

    def __call__(self, cam, render_pkg, iteration):
        assert "raw_depth" in render_pkg, "Forgot to set `output_depth=True` when calling render?"
        assert "raw_normal" in render_pkg, "Forgot to set `output_normal=True` when calling render?"
        if not self.is_active(iteration):
            return 0
        T = render_pkg.get("raw_T")
        T = render_pkg["raw_depth"][0:1].detach() if T is None else T.detach()
        return _NormalLoss.apply(render_pkg["raw_depth"], render_pkg["raw_normal"], T, cam, "dmed", 3, -1.0)
