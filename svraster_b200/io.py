"""Checkpoint and scene formats: drop-in for src/sparse_voxel_gears/io.py and the
checkpoint half of src/sparse_voxel_gears/optimizer.py.

A checkpoint is the reference's file, byte-compatible in structure: ``torch.save`` of a dict
with keys active_sh_degree, ss, scene_center, inside_extent, scene_extent, octpath,
octlevel, _geo_grid_pts, _sh0, _shs, _log_s, is_leaf and quantized (io.py:23-42).  With
``quantize=True`` the SDF grid becomes one {index u8, codebook f32[256]} dict and sh0 / shs
become lists of such dicts, one per column of dim 1 (io.py:111-121).  Files written by the
reference load here and files written here load in the reference.  The codebook is built by
the sm_100a library (``svr_quantize``); on load the library rebuilds voxel centres, sizes and
the corner grid-point link from the octree paths (``svr_grid_link``).

``dump_config`` / ``load_config`` keep the run's ``config.yaml`` (train.py:1381-1383): the
reference writes yacs ``CfgNode.dump()``, which is ``yaml.safe_dump`` of the nested
dictionary with PyYAML's defaults.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import torch

from . import _lib
from ._lib import check, ptr, stream_ptr
from . import adaptive

STATE_KEYS = ("active_sh_degree", "ss", "scene_center", "inside_extent", "scene_extent", "octpath", "octlevel",
              "_geo_grid_pts", "_sh0", "_shs", "_log_s", "is_leaf")


def _device():
    if not torch.cuda.is_available():
        raise RuntimeError("svraster_b200.io needs a CUDA device (the codebook and the grid link are built "
                           "by the sm_100a library)")
    return torch.device("cuda", torch.cuda.current_device())


def quantization(src_tensor, max_iter=10):
    """io.py:123-167: {index: u8 tensor shaped like src_tensor, codebook: f32[256]} on the
    input's device.  Raises for an empty tensor (the reference fails on one too)."""
    src_dev = src_tensor.device
    dev = src_dev if src_dev.type == "cuda" else _device()
    vals = src_tensor.detach().reshape(-1).to(dev, torch.float32).contiguous()
    n = vals.numel()
    L = _lib.load()
    nbytes = C.c_size_t(0)
    check(L.svr_quantize_workspace_bytes(n, C.byref(nbytes)), "svr_quantize_workspace_bytes")
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    index = torch.empty(n, dtype=torch.uint8, device=dev)
    book = torch.empty(256, dtype=torch.float32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    rounds = C.c_int(0)
    check(L.svr_quantize(n, ptr(vals), int(max_iter), ptr(index), ptr(book), ptr(ws), nbytes.value,
                         C.byref(rounds), ptr(status), stream_ptr(dev)), "svr_quantize")
    if int(status.item()):
        raise ValueError("quantization: the tensor holds non-finite values")
    return dict(index=index.reshape(src_tensor.shape).to(src_dev), codebook=book.to(src_dev))


def dequantization(quant_dict):
    """io.py:169-170: codebook[index] as float32, on the index's device (GPU when it is on
    the CPU and a GPU is present the work runs there and the result comes back)."""
    index, book = quant_dict["index"], quant_dict["codebook"]
    src_dev = index.device
    dev = src_dev if src_dev.type == "cuda" else _device()
    idx = index.to(dev, torch.uint8).contiguous()
    cb = book.to(dev, torch.float32).contiguous()
    if cb.numel() != 256:
        raise ValueError("dequantization: the codebook must hold 256 entries")
    out = torch.empty(idx.shape, dtype=torch.float32, device=dev)
    check(_lib.load().svr_dequantize(idx.numel(), ptr(idx), ptr(cb), ptr(out), stream_ptr(dev)), "svr_dequantize")
    return out.to(src_dev)


def quantize_state_dict(state_dict):
    """io.py:111-114: in place; sh0 / shs quantized per column of dim 1."""
    state_dict["_geo_grid_pts"] = quantization(state_dict["_geo_grid_pts"])
    state_dict["_sh0"] = [quantization(v) for v in state_dict["_sh0"].split(1, dim=1)]
    state_dict["_shs"] = [quantization(v) for v in state_dict["_shs"].split(1, dim=1)]


def dequantize_state_dict(state_dict):
    """io.py:116-121: in place."""
    state_dict["_geo_grid_pts"] = dequantization(state_dict["_geo_grid_pts"])
    state_dict["_sh0"] = torch.cat([dequantization(v) for v in state_dict["_sh0"]], dim=1)
    state_dict["_shs"] = torch.cat([dequantization(v) for v in state_dict["_shs"]], dim=1)


def read_state_dict(path):
    """The checkpoint's dict with quantized fields expanded, tensors on the CPU.  Loads with
    ``weights_only=True``: a checkpoint holds only tensors, numbers, lists and dicts."""
    state_dict = torch.load(path, map_location="cpu", weights_only=True)
    if state_dict.get("quantized", False):
        dequantize_state_dict(state_dict)
    return state_dict


class SVInOut:
    """Mixin with the reference model's save / load (io.py:16-106)."""

    def save(self, path, quantize=False):
        """io.py:18-48."""
        d = os.path.dirname(path)
        if d:
            os.makedirs(d, exist_ok=True)
        state_dict = {}
        for k in STATE_KEYS:
            v = getattr(self, k)
            state_dict[k] = v.data.contiguous() if torch.is_tensor(v) else v
        if quantize:
            quantize_state_dict(state_dict)
        state_dict["quantized"] = bool(quantize)
        for k, v in state_dict.items():
            if torch.is_tensor(v):
                state_dict[k] = v.cpu()
            elif isinstance(v, dict):
                state_dict[k] = {kk: vv.cpu() for kk, vv in v.items()}
            elif isinstance(v, list):
                state_dict[k] = [{kk: vv.cpu() for kk, vv in q.items()} for q in v]
        torch.save(state_dict, path)
        self.latest_save_path = path

    def load(self, path):
        """io.py:50-86: fields on the current GPU, voxel centres / sizes and the grid-point
        link rebuilt from the octree paths, _subdiv_p = 1 and subdiv_meta = 0 per voxel."""
        dev = _device()
        state_dict = read_state_dict(path)
        self.active_sh_degree = state_dict["active_sh_degree"]
        self.ss = state_dict["ss"]
        self.scene_center = state_dict["scene_center"].to(dev)
        self.inside_extent = state_dict["inside_extent"].to(dev)
        self.scene_extent = state_dict["scene_extent"].to(dev)
        self.octpath = state_dict["octpath"].to(dev)
        self.octlevel = state_dict["octlevel"].to(dev).to(torch.int8)
        self.vox_center, self.vox_size = adaptive.octpath_decoding(self.octpath, self.octlevel, self.scene_center,
                                                                   self.scene_extent)
        self.grid_pts_key, self.vox_key = adaptive.build_grid_pts_link(self.octpath, self.octlevel)
        self._geo_grid_pts = state_dict["_geo_grid_pts"].to(dev).requires_grad_()
        self._sh0 = state_dict["_sh0"].to(dev).requires_grad_()
        self._shs = state_dict["_shs"].to(dev).requires_grad_()
        self._log_s = state_dict["_log_s"].to(dev).requires_grad_()
        self.is_leaf = state_dict["is_leaf"].to(dev)
        N = len(self.octpath)
        self._subdiv_p = torch.full([N, 1], 1.0, dtype=torch.float32, device=dev).requires_grad_()
        self.subdiv_meta = torch.zeros([N, 1], dtype=torch.float32, device=dev)
        white = getattr(self, "white_background", False)
        self.bg_color = torch.tensor([1, 1, 1] if white else [0, 0, 0], dtype=torch.float32, device=dev)
        self.loaded_path = path

    def save_iteration(self, iteration, quantize=False):
        """io.py:88-91: <model_path>/checkpoints/iterNNNNNN_model.pt."""
        self.save(os.path.join(self.model_path, "checkpoints", f"iter{iteration:06d}_model.pt"), quantize=quantize)
        self.latest_save_iter = iteration

    def load_iteration(self, iteration=-1):
        """io.py:93-106: iteration -1 loads the highest-numbered model checkpoint."""
        if iteration == -1:
            fnames = os.listdir(os.path.join(self.model_path, "checkpoints"))
            loaded_iter = max(int(re.sub("[^0-9]", "", f)) for f in fnames)
        else:
            loaded_iter = iteration
        self.load(os.path.join(self.model_path, "checkpoints", f"iter{loaded_iter:06d}_model.pt"))
        self.loaded_iter = iteration
        return loaded_iter


class SVOptimizerIO:
    """Mixin with the optimiser checkpoint of src/sparse_voxel_gears/optimizer.py:29-45:
    {'optimizer': self.optimizer.state_dict()} in iterNNNNNN_optim.pt (the state of
    svraster_b200.sparse_adam.SparseAdam has the reference's keys: step, exp_avg,
    exp_avg_sq)."""

    def optimizer_save(self, path):
        d = os.path.dirname(path)
        if d:
            os.makedirs(d, exist_ok=True)
        torch.save({"optimizer": self.optimizer.state_dict()}, path)

    def optimizer_load(self, path):
        state_dict = torch.load(path, map_location=_device(), weights_only=True)
        self.optimizer.load_state_dict(state_dict["optimizer"])

    def optimizer_save_iteration(self, iteration):
        self.optimizer_save(os.path.join(self.model_path, "checkpoints", f"iter{iteration:06d}_optim.pt"))

    def optimizer_load_iteration(self, iteration):
        self.optimizer_load(os.path.join(self.model_path, "checkpoints", f"iter{iteration:06d}_optim.pt"))


def _plain(cfg):
    if isinstance(cfg, dict):
        return {str(k): _plain(v) for k, v in cfg.items()}
    if isinstance(cfg, tuple):
        return [_plain(v) for v in cfg]
    if isinstance(cfg, list):
        return [_plain(v) for v in cfg]
    return cfg


def dump_config(cfg, path=None):
    """The text of config.yaml for a nested configuration (dicts, yacs CfgNode included):
    ``yaml.safe_dump`` with PyYAML's defaults, as CfgNode.dump() writes it.  Written to
    ``path`` when given."""
    import yaml
    text = yaml.safe_dump(_plain(cfg))
    if path is not None:
        with open(path, "w") as f:
            f.write(text)
    return text


def load_config(path):
    """A config.yaml (this module's or the reference's) as nested dicts."""
    import yaml
    with open(path) as f:
        return yaml.safe_load(f)
