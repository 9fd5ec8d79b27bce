"""The reference's own callers on top of the drop-in package (CPU; needs the reference checkout
on this machine, given by SVR_REFERENCE_DIR; skipped where it is absent).

* Every ``svraster_cuda.<module>.<name>(...)`` call in the reference's Python callers
  (train.py, extract_mesh_sdf.py, src/**) names something the drop-in package exports, and
  its positional / keyword arguments bind to that function's signature.
* ``SVRenderer.render`` from src/sparse_voxel_gears/renderer.py runs unchanged on the
  package installed as ``svraster_cuda``: the settings it builds and the arguments it passes
  pass every check of ``rasterize_voxels`` and reach the native boundary, where the package
  refuses host tensors (there is no GPU here and no CPU fallback).
"""
from __future__ import annotations

import ast
import inspect
import os
import sys

import pytest
import torch

REF = os.environ.get("SVR_REFERENCE_DIR") or "/root/reference"
pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src", "sparse_voxel_gears")),
                                reason="reference checkout not present")


def _caller_files():
    out = [os.path.join(REF, f) for f in ("train.py", "extract_mesh_sdf.py") if os.path.exists(os.path.join(REF, f))]
    for root, _, files in os.walk(os.path.join(REF, "src")):
        out += [os.path.join(root, f) for f in files if f.endswith(".py")]
    return sorted(out)


def _call_sites(path):
    """(module, name, n_positional, keyword names, has_star) of every svraster_cuda.m.f(...) call."""
    tree = ast.parse(open(path).read(), path)
    sites = []
    for node in ast.walk(tree):
        if not isinstance(node, ast.Call):
            continue
        f = node.func
        # svraster_cuda.mod.fn(...) or svraster_cuda.mod.Class.apply(...)
        chain = []
        while isinstance(f, ast.Attribute):
            chain.append(f.attr)
            f = f.value
        if not (isinstance(f, ast.Name) and f.id == "svraster_cuda") or len(chain) < 2:
            continue
        chain = chain[::-1]
        star = any(isinstance(a, ast.Starred) for a in node.args) or any(k.arg is None for k in node.keywords)
        sites.append((chain, len(node.args), [k.arg for k in node.keywords if k.arg], star, node.lineno))
    return sites


def test_every_reference_call_site_binds_to_the_package():
    import svraster_b200
    pkg = svraster_b200
    checked = 0
    for path in _caller_files():
        for chain, n_pos, kws, star, line in _call_sites(path):
            obj = pkg
            for part in chain:
                assert hasattr(obj, part), f"{os.path.relpath(path, REF)}:{line}: svraster_cuda.{'.'.join(chain)} missing"
                obj = getattr(obj, part)
            if star:
                continue
            if chain[-1] == "apply":          # autograd Function: bind against forward(ctx, ...)
                sig = inspect.signature(getattr(pkg, chain[0]).__dict__[chain[1]].forward)
                n_pos += 1
            else:
                sig = inspect.signature(obj)
            try:
                sig.bind(*range(n_pos), **{k: None for k in kws})
            except TypeError as e:
                pytest.fail(f"{os.path.relpath(path, REF)}:{line}: svraster_cuda.{'.'.join(chain)}{sig}: {e}")
            checked += 1
    assert checked >= 20, checked


class _Camera:
    """The camera fields SVRenderer.render reads (src/cameras.py)."""

    def __init__(self, W=64, H=48):
        from svraster_b200 import synthetic as S
        c = S.look_at_camera([2.5, 1.0, 0.8], W, H)
        self.image_width, self.image_height = W, H
        self.tanfovx, self.tanfovy = c.tanfovx, c.tanfovy
        self.cx, self.cy = c.cx, c.cy
        self.w2c = torch.as_tensor(c.w2c)
        self.c2w = torch.as_tensor(c.c2w)
        self.cam_mode = "persp"
        self.near = c.near


def test_reference_renderer_runs_unchanged_up_to_the_native_boundary():
    import svraster_b200
    from svraster_b200 import synthetic as S
    from svraster_b200._lib import SvrError
    svraster_b200.install_as_svraster_cuda()
    if REF not in sys.path:
        sys.path.insert(0, REF)
    from src.sparse_voxel_gears.renderer import SVRenderer   # the reference's module, unmodified

    sc = S.scene_tiny(seed=0)
    t = lambda a, dt=torch.float32: torch.as_tensor(a).to(dt)

    class Model(SVRenderer):
        pass
    m = Model()
    m.vox_geo_mode, m.density_mode, m.ss = "triinterp3", "sdf", 1.0
    m.white_background, m.black_background = False, True
    m.octpath = t(sc.octpath.reshape(-1, 1), torch.int64)
    m.vox_center, m.vox_size = t(sc.vox_center), t(sc.vox_size)
    m.is_leaf = t(sc.is_leaf.reshape(-1, 1), torch.bool)
    m.vox_key, m._geo_grid_pts = t(sc.vox_key, torch.int64), t(sc.geo_grid_pts)
    m.vox_size_inv = 1.0 / m.vox_size
    m.sh0, m.shs, m.active_sh_degree = t(sc.sh0), t(sc.shs), 3
    m._subdiv_p = torch.zeros(sc.n_vox, 1)
    m._log_s = torch.tensor([sc.log_s])
    m.bg_color = torch.zeros(3)
    m.num_voxels = sc.n_vox
    with pytest.raises(SvrError, match="CUDA tensors"):
        m.render(_Camera(), output_depth=True, output_normal=True, output_T=True)
