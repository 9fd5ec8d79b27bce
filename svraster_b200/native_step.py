"""The batched training step driven through the library's native step object (svr_step_*).

``NativeStep`` hands the octree and the parameters to ``svr_step_create`` and lets the
library run the whole step: the same launches as ``step.BatchedTrainStep`` (gather, SH of
every view, preprocess, per-tile binning, render forward and adjoint, fused smoothness
adjoint, gradient scatter, SH adjoint, Adam), issued and graph-captured by the library's own
host code instead of Python.  It is what a non-Python host sees through the C ABI; Python only
owns the parameter tensors and reads the step's buffers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check, stream_ptr

BUFFERS = {"color": 0, "depth": 1, "normal": 2, "T": 3, "dcolor": 4, "ddepth": 5, "dnormal": 6, "dT": 7, "gt": 8,
           "grad_flat": 9, "grad_grid": 10, "grad_sh0": 11, "grad_shs": 12, "dvox": 13, "ds": 14, "step": 15}
GRADS, ADAM = 1, 2


class _DeviceArray:
    """A step-owned device buffer exposed to torch without a copy (CUDA array interface)."""

    def __init__(self, ptr, n, typestr, owner):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}
        self._owner = owner


class NativeStep:
    """One native step object over a scene (``synthetic.Scene``-like: octpath, vox_center,
    vox_size, is_leaf, vox_key, geo_grid_pts, sh0, shs, s_val, octlevel, scene_extent) and a
    list of cameras.  Arguments as ``step.BatchedTrainStep`` (the smoothness grid resolution
    is min(finest level, 9), as there)."""

    def __init__(self, scene, cams, device="cuda", lr=(1e-3, 1e-3, 1e-4), betas=(0.1, 0.99), eps=1e-15,
                 lambda_ls=1e-3, lambda_ge=1e-3, lambda_R_concen=0.0, sh_degree=3, seed=0, sh_dtype="f32",
                 record_capacity=0, adam_rows=0):
        if sh_dtype not in ("f32", "bf16"):
            raise ValueError("sh_dtype must be 'f32' or 'bf16'")
        dev = torch.device(device)
        self.dev = dev
        t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt).contiguous()
        self.N = int(scene.n_vox)
        self.octpath = t(scene.octpath, torch.int64)
        self.centers = t(scene.vox_center)
        self.lengths = t(scene.vox_size).reshape(-1).contiguous()
        self.is_leaf = t(scene.is_leaf, torch.uint8)
        self.vox_key = t(scene.vox_key, torch.int64)
        self.grid = t(scene.geo_grid_pts)
        sh_t = torch.bfloat16 if sh_dtype == "bf16" else torch.float32
        self.sh0 = t(scene.sh0).to(sh_t).contiguous()
        self.shs = t(scene.shs).to(sh_t).contiguous()
        self.s_val = torch.tensor([scene.s_val], dtype=torch.float32, device=dev)
        self.cams = [dict(width=c.width, height=c.height, tanfovx=c.tanfovx, tanfovy=c.tanfovy, cx=c.cx, cy=c.cy,
                          near=c.near, w2c=t(c.w2c), c2w=t(c.c2w), bg=torch.zeros(3, device=dev)) for c in cams]
        views, _, _ = _lib.make_views(self.cams)
        d = _lib.StepDesc()
        d.n_vox, d.sh_degree, d.sh_bf16 = self.N, int(sh_degree), int(sh_dtype == "bf16")
        d.grid_res_pow2 = min(int(np.asarray(scene.octlevel).max()), 9)
        for name in ("octpath", "centers", "lengths", "is_leaf", "vox_key", "grid", "sh0", "shs", "s_val"):
            setattr(d, name, getattr(self, name).data_ptr())
        d.n_grid = self.grid.numel()
        d.scene_center[:] = (0.0, 0.0, 0.0)
        d.inside_extent = float(scene.scene_extent)
        d.lambda_ls, d.lambda_ge, d.lambda_R_concen = float(lambda_ls), float(lambda_ge), float(lambda_R_concen)
        d.lr[:] = tuple(float(x) for x in lr)
        d.beta1, d.beta2, d.eps = float(betas[0]), float(betas[1]), float(eps)
        d.seed, d.adam_rows, d.record_capacity = int(seed), int(adam_rows), int(record_capacity)
        self.desc = d
        L = _lib.load()
        h = C.c_void_p()
        check(L.svr_step_create(C.byref(d), views, len(self.cams), stream_ptr(dev), C.byref(h)), "svr_step_create")
        self.handle = h
        self._bufs = {}

    # ------------------------------------------------------------------ buffers
    def buffer(self, name):
        """A step-owned buffer as a flat torch tensor sharing its memory (see BUFFERS)."""
        b = self._bufs.get(name)
        if b is None:
            p, n = C.c_void_p(), C.c_int64()
            check(_lib.load().svr_step_buffer(self.handle, BUFFERS[name], C.byref(p), C.byref(n)), "svr_step_buffer")
            if not p.value or n.value == 0:
                return None
            typestr = "<i8" if name == "step" else "<f4"
            b = self._bufs[name] = torch.as_tensor(_DeviceArray(p.value, n.value, typestr, self), device=self.dev)
        return b

    def info(self):
        out = (C.c_int64 * 8)()
        check(_lib.load().svr_step_info(self.handle, out), "svr_step_info")
        keys = ("pixels", "capacity", "tiles", "grid_rows", "grad_flat", "views", "kernels", "captured")
        return dict(zip(keys, (int(x) for x in out)))

    # ------------------------------------------------------------------ stepping
    def run(self, phases=GRADS | ADAM):
        check(_lib.load().svr_step_run(self.handle, int(phases), stream_ptr(self.dev)), "svr_step_run")

    def capture(self):
        check(_lib.load().svr_step_capture(self.handle, stream_ptr(self.dev)), "svr_step_capture")
        return self.info()["kernels"]

    def status(self):
        r, o = C.c_uint32(), C.c_uint32()
        check(_lib.load().svr_step_status(self.handle, C.byref(r), C.byref(o), stream_ptr(self.dev)), "svr_step_status")
        return int(r.value), int(o.value)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            torch.cuda.synchronize(self.dev)
            self._bufs.clear()
            _lib.load().svr_step_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
