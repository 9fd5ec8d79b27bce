"""The native batched step (svr_step_*): the same step as the Python orchestration
(``step.BatchedTrainStep``) issued by the library's own host code, eagerly and as CUDA graphs,
and from a host program in plain C (``tests/native_host/step_driver.c``, no Python in that
process).

The render adjoint accumulates with float atomics, so two runs of the same step agree on the
forward planes bit for bit and on the gradients up to the order of those additions.  Adam's
first step moves every parameter with a non-zero gradient by lr * g / (|g| + eps), i.e. by
+-lr: after one step the parameters agree exactly except where a gradient that is zero up to
rounding takes another sign, which the tolerance below allows for a few elements."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest
import torch

from svraster_b200.native_step import NativeStep
from svraster_b200.step import BatchedTrainStep
from tests import native_host
from tests.helpers import scene_and_cams

pytestmark = pytest.mark.gpu

HYPER = dict(lr=(1e-3, 1e-3, 1e-4), betas=(0.1, 0.99), eps=1e-15, lambda_ls=1e-3, lambda_ge=1e-3, seed=5)


@pytest.fixture(scope="module")
def scene():
    return scene_and_cams("small", n_cams=3, W=200, H=150)


def _grad_close(a, b, rel=1e-5):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    assert np.abs(a - b).max() <= rel * scale, (np.abs(a - b).max(), scale)


def _params_close(a, b, lr, frac=1e-3):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    d = np.abs(a - b)
    assert d.max() <= 2.0 * lr * (1 + 1e-3) + 1e-6 * np.abs(b).max()
    assert (d > 1e-3 * lr).mean() <= frac


def _python_step(sc, cams):
    bts = BatchedTrainStep(sc, cams, lr=HYPER["lr"], betas=HYPER["betas"], eps=HYPER["eps"],
                           lambda_ls=HYPER["lambda_ls"], lambda_ge=HYPER["lambda_ge"], seed=HYPER["seed"])
    return bts


def _native(sc, cams, **kw):
    return NativeStep(sc, cams, lr=HYPER["lr"], betas=HYPER["betas"], eps=HYPER["eps"], lambda_ls=HYPER["lambda_ls"],
                      lambda_ge=HYPER["lambda_ge"], seed=HYPER["seed"], **kw)


def _load_upstream(ns, bts):
    for name in ("dcolor", "ddepth", "dnormal"):
        ns.buffer(name).copy_(getattr(bts, name))


def test_native_step_matches_python_step(scene):
    sc, cams = scene
    bts = _python_step(sc, cams)
    ns = _native(sc, cams)
    _load_upstream(ns, bts)
    info = ns.info()
    assert info["pixels"] == bts.P and info["views"] == len(cams)
    color_p, T_p = bts.step()
    ns.run()
    torch.cuda.synchronize()
    assert info["capacity"] == bts.state.num_rendered
    assert ns.status() == (0, 0)
    # forward planes: bit for bit
    assert torch.equal(ns.buffer("color"), color_p) and torch.equal(ns.buffer("T"), T_p)
    # gradients (atomics) and the parameters after Adam
    for k, name in enumerate(("grad_grid", "grad_sh0", "grad_shs")):
        _grad_close(ns.buffer(name).cpu().numpy(), bts.grads[k].reshape(-1).cpu().numpy())
    _grad_close(ns.buffer("dvox").cpu().numpy(), bts.dvox.reshape(-1).cpu().numpy())
    for k, (a, b) in enumerate(((ns.grid, bts.grid), (ns.sh0, bts.sh0), (ns.shs, bts.shs))):
        _params_close(a.cpu().numpy(), b.cpu().numpy(), HYPER["lr"][k])
    assert int(ns.buffer("step").item()) == 1
    # the gradient views sit in the flat buffer on 256-byte boundaries
    flat = ns.buffer("grad_flat")
    for name in ("grad_grid", "grad_sh0", "grad_shs"):
        off = (ns.buffer(name).data_ptr() - flat.data_ptr())
        assert off % 256 == 0 and 0 <= off < 4 * flat.numel()
    ns.close()


def test_native_graph_matches_native_eager(scene):
    sc, cams = scene
    bts = _python_step(sc, cams)     # the upstream planes only
    eager, graph = _native(sc, cams), _native(sc, cams)
    _load_upstream(eager, bts)
    _load_upstream(graph, bts)
    k = graph.capture()
    assert k >= 12 and graph.info()["captured"] == 1
    # capture ran the gradient phase once but no Adam step
    assert int(graph.buffer("step").item()) == 0
    torch.testing.assert_close(graph.grid, eager.grid, rtol=0, atol=0)
    for it in range(3):
        eager.run()
        graph.run()
        torch.cuda.synchronize()
        if it == 0:
            assert torch.equal(eager.buffer("color"), graph.buffer("color"))
            _grad_close(graph.buffer("grad_flat").cpu().numpy(), eager.buffer("grad_flat").cpu().numpy())
    assert int(graph.buffer("step").item()) == 3 and int(eager.buffer("step").item()) == 3
    assert graph.status() == (0, 0) and eager.status() == (0, 0)
    # three steps apart only by the atomics' rounding and rare first-step sign flips
    c_e, c_g = eager.buffer("color").cpu().numpy(), graph.buffer("color").cpu().numpy()
    assert np.percentile(np.abs(c_e - c_g), 99.9) < 1e-4
    # phases run apart: gradients, then Adam, as a data-parallel host would with its all-reduce
    before = graph.grid.clone()
    graph.run(1)
    torch.cuda.synchronize()
    assert torch.equal(graph.grid, before) and int(graph.buffer("step").item()) == 3
    graph.run(2)
    torch.cuda.synchronize()
    assert not torch.equal(graph.grid, before) and int(graph.buffer("step").item()) == 4
    eager.close()
    graph.close()


@pytest.mark.parametrize("mode", ["eager", "graph"])
def test_plain_c_host_drives_the_step(scene, tmp_path, mode):
    sc, cams = scene
    bts = _python_step(sc, cams)
    up = [getattr(bts, n).cpu().numpy() for n in ("dcolor", "ddepth", "dnormal")]
    hyper = dict(HYPER, sh_degree=3, grid_res_pow2=min(int(np.asarray(sc.octlevel).max()), 9))
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    native_host.write_input(inp, sc, cams, up, hyper)
    exe = native_host.compile_driver(str(tmp_path))
    env = dict(os.environ)
    r = subprocess.run([exe, inp, out, "1", mode], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr
    N, M = sc.n_vox, 16
    res = native_host.read_output(out, bts.P, sc.geo_grid_pts.size, N, M)
    assert int(res["info"][6]) >= 12 and tuple(res["status"]) == (0, 0)
    color_p, T_p = bts.step()
    torch.cuda.synchronize()
    assert int(res["info"][1]) == bts.state.num_rendered
    assert np.array_equal(res["color"], color_p.cpu().numpy()) and np.array_equal(res["T"], T_p.cpu().numpy())
    flat = res["grad_flat"]
    n_grid = sc.geo_grid_pts.size
    _grad_close(flat[:n_grid], bts.grads[0].reshape(-1).cpu().numpy())
    for got, ref, lr in ((res["grid"], bts.grid, HYPER["lr"][0]), (res["sh0"], bts.sh0, HYPER["lr"][1]),
                         (res["shs"], bts.shs, HYPER["lr"][2])):
        _params_close(got, ref.cpu().numpy(), lr)
