"""The allocation-free Laplacian adjoint (svr_laplacian_bw_noalloc).

Some callers cannot allocate device memory themselves, for instance a host application that
reserves all device memory in a fixed arena when it starts and forbids cudaMalloc later.
For them the library keeps the adjoint's key-index scratch in a static device array.  This
test calls that entry point through the C ABI twice in a row and checks each result against
the regular entry point (svr_laplacian_bw, index scratch supplied by the caller) on the same
inputs and seed.  The file is named so pytest collects it last.
"""
import numpy as np
import pytest
import torch

from svraster_b200 import _lib, utils
from svraster_b200 import synthetic as S
from svraster_b200._lib import check, ptr, stream_ptr
from tests.golden.cases import grid_voxel_geometry

pytestmark = pytest.mark.gpu


def _inputs():
    dev = torch.device("cuda")
    sc = S.scene_small(seed=5)
    res_pow2 = 7
    res = 1 << res_pow2
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    centers, sizes = t(sc.vox_center), t(sc.vox_size)
    mask, keys, g2v = utils.valid_gradient_table(centers, sizes, t(np.zeros(3)), sc.scene_extent, res_pow2,
                                                 t(sc.is_leaf, torch.uint8))
    coord, vsize = grid_voxel_geometry(sc, res_pow2)
    rng = np.random.default_rng(11)
    active = rng.permutation(keys.numel())[: keys.numel() // 2].astype(np.int32)
    return dict(sc=sc, res=res, mask=mask.contiguous(), keys=keys.contiguous(), g2v=g2v.contiguous(),
                coord=t(coord), vsize=t(vsize), active=t(active, torch.int32), vox_key=t(sc.vox_key, torch.int64),
                grid=t(sc.geo_grid_pts))


def _run(fn_name, d, seed, with_index):
    L = _lib.load()
    grad = torch.zeros_like(d["grid"])
    status = torch.zeros(1, dtype=torch.int32, device=grad.device)
    common = (d["keys"].numel(), d["active"].numel(), ptr(d["active"]), ptr(d["keys"]), ptr(d["g2v"]), d["res"],
              ptr(d["mask"]))
    tail = (ptr(d["coord"]), ptr(d["vsize"]), d["sc"].n_vox, ptr(d["vox_key"]), ptr(d["grid"]), d["grid"].numel(),
            0.01, float(d["res"]) / d["sc"].scene_extent, seed, ptr(grad), ptr(status), stream_ptr())
    if with_index:
        check(getattr(L, fn_name)(*common, None, *tail), fn_name)
    else:
        check(getattr(L, fn_name)(*common, *tail), fn_name)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return grad.cpu().numpy()


def _half_table(d):
    """Every second key of the grid table with its voxel row, and a fresh active set over it:
    if the shared index kept entries of an earlier call, they would point at wrong rows."""
    out = dict(d)
    out["keys"] = d["keys"][::2].contiguous()
    out["g2v"] = d["g2v"][::2].contiguous()
    rng = np.random.default_rng(12)
    G = out["keys"].numel()
    out["active"] = torch.as_tensor(rng.permutation(G)[: G // 2].astype(np.int32), device=d["grid"].device)
    return out


def test_noalloc_laplacian_matches_regular_entry_point_twice():
    d = _inputs()
    # two calls in a row, the second on a smaller key table: the shared index must be rebuilt
    for inputs, seed in ((d, 123), (_half_table(d), 456)):
        got = _run("svr_laplacian_bw_noalloc", inputs, seed, with_index=False)
        ref = _run("svr_laplacian_bw", inputs, seed, with_index=True)
        scale = np.abs(ref).max()
        assert scale > 0
        # same arithmetic; only the order of the float atomics differs
        assert np.abs(got - ref).max() <= 1e-5 * scale + 1e-7


def test_noalloc_rejects_grid_beyond_static_capacity():
    d = _inputs()
    L = _lib.load()
    grad = torch.zeros_like(d["grid"])
    status = torch.zeros(1, dtype=torch.int32, device=grad.device)
    rc = L.svr_laplacian_bw_noalloc(d["keys"].numel(), d["active"].numel(), ptr(d["active"]), ptr(d["keys"]),
                                    ptr(d["g2v"]), 256, ptr(d["mask"]), ptr(d["coord"]), ptr(d["vsize"]),
                                    d["sc"].n_vox, ptr(d["vox_key"]), ptr(d["grid"]), d["grid"].numel(), 0.01, 1.0, 1,
                                    ptr(grad), ptr(status), stream_ptr())
    assert rc == -3
    assert b"capacity" in L.svr_last_error()


def test_noalloc_rejects_null_arguments_before_any_launch():
    d = _inputs()
    L = _lib.load()
    grad = torch.zeros_like(d["grid"])
    status = torch.zeros(1, dtype=torch.int32, device=grad.device)
    args = [d["keys"].numel(), d["active"].numel(), ptr(d["active"]), ptr(d["keys"]), ptr(d["g2v"]), d["res"],
            ptr(d["mask"]), ptr(d["coord"]), ptr(d["vsize"]), d["sc"].n_vox, ptr(d["vox_key"]), ptr(d["grid"]),
            d["grid"].numel(), 0.01, 1.0, 1, ptr(grad), ptr(status), stream_ptr()]
    for i in (3, 4, 16, 17):            # grid_keys, grid2voxel, grid_grad, status
        bad = list(args)
        bad[i] = None
        assert L.svr_laplacian_bw_noalloc(*bad) == -1
    bad = list(args)
    bad[5] = 0                          # grid_res <= 0 is a bad argument, not a capacity problem
    assert L.svr_laplacian_bw_noalloc(*bad) == -1
    torch.cuda.synchronize()
    assert float(grad.abs().sum()) == 0.0
