"""The product path has no CPU fallback: every public entry point given host tensors raises
instead of computing (the CUDA library is the only implementation; the CPU restatement under
oracle/ is test infrastructure and never called by the package)."""
import ast
import os

import pytest
import torch

from svraster_b200 import grid_loss_bw, marching_cubes, renderer, utils
from svraster_b200._lib import SvrError
from svraster_b200.sparse_adam import SparseAdam

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _vox(n=4):
    return dict(octpath=torch.arange(n, dtype=torch.int64).view(-1, 1),
                centers=torch.rand(n, 3), lengths=torch.full((n, 1), 0.25),
                vox_key=torch.arange(8 * n, dtype=torch.int64).view(n, 8), grid=torch.rand(8 * n, 1))


def test_gather_and_sh_refuse_host_tensors():
    v = _vox()
    with pytest.raises(SvrError):
        renderer.GatherGeoParams.apply("triinterp3", v["vox_key"], 1.0, torch.arange(4), v["grid"])
    with pytest.raises(SvrError):
        renderer.SH_eval.apply(3, None, v["centers"], torch.zeros(3), None, torch.rand(4, 3), torch.rand(4, 15, 3))


def test_regularisers_and_extraction_refuse_host_tensors():
    v = _vox()
    grad = torch.zeros_like(v["grid"])
    vsi = torch.full((4,), 4.0)
    with pytest.raises(SvrError):
        grid_loss_bw.total_variation(v["grid"], v["vox_key"], 1.0, vsi, False, False, grad)
    with pytest.raises(SvrError):
        grid_loss_bw.voxel_gradient(v["grid"], v["vox_key"], vsi, torch.arange(4), 1.0, False, False, grad)
    with pytest.raises(SvrError):
        marching_cubes.torch_marching_cubes_grid(v["grid"], torch.rand(8 * 4, 3), v["vox_key"], 0.0)
    with pytest.raises(SvrError):
        utils.valid_gradient_table(v["centers"], v["lengths"], torch.zeros(3), 2.0, 4, torch.ones(4, 1))


def test_optimizer_refuses_host_parameters():
    p = torch.nn.Parameter(torch.rand(8, 3))
    p.grad = torch.ones_like(p)
    opt = SparseAdam([p], lr=0.1)
    with pytest.raises(SvrError):
        opt.step()
    assert torch.equal(p.grad, torch.ones_like(p))


def test_package_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "svraster_b200")
    for dp, _, files in os.walk(pkg):
        for f in files:
            if not f.endswith(".py"):
                continue
            tree = ast.parse(open(os.path.join(dp, f)).read())
            for node in ast.walk(tree):
                mods = []
                if isinstance(node, ast.Import):
                    mods = [a.name for a in node.names]
                elif isinstance(node, ast.ImportFrom):
                    mods = [node.module or ""]
                assert not any(m == "oracle" or m.startswith("oracle.") for m in mods), (f, mods)
