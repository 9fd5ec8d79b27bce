"""Normal-from-depth consistency losses on the GPU (``svr_normal_depth_loss`` through the
drop-in ``svraster_b200.loss_utils`` classes and the batched form) against the reference's
own torch code (tests/golden/nd_*.npz) and, at 800x800 and over packed multi-view planes,
against the C oracle."""
from __future__ import annotations

import os
import types

import numpy as np
import pytest
import torch

from svraster_b200 import loss_utils as LU
from svraster_b200 import synthetic as S
from tests.golden.nd_cases import ND_CASES, nd_camera, nd_inputs
from tests.test_losses_cpu import GRAD_TOL, LOSS_RTOL

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def ref_style_camera(cam, c2w):
    return types.SimpleNamespace(image_width=cam.width, image_height=cam.height, cx=cam.cx, cy=cam.cy,
                                 tanfovx=cam.tanfovx, tanfovy=cam.tanfovy, c2w=torch.from_numpy(c2w).cuda())


@pytest.mark.parametrize("name", list(ND_CASES))
def test_dropin_loss_matches_reference(name):
    case = ND_CASES[name]
    g = np.load(os.path.join(HERE, f"nd_{name}.npz"))
    depth, normal, T = nd_inputs(case, g["c2w"])
    d = torch.from_numpy(depth).cuda().requires_grad_()
    n = torch.from_numpy(normal).cuda().requires_grad_()
    pkg = {"raw_depth": d, "raw_normal": n, "raw_T": torch.from_numpy(T).cuda()}
    if case["mode"] == "dmean":
        fn = LU.NormalDepthConsistencyLoss(iter_from=0, iter_end=10, ks=case["ks"], tol_deg=case["tol_deg"])
    else:
        fn = LU.NormalMedianConsistencyLoss(iter_from=0, iter_end=10)
    assert fn(ref_style_camera(nd_camera(case), g["c2w"]), pkg, 20) == 0      # inactive outside its window
    loss = fn(ref_style_camera(nd_camera(case), g["c2w"]), pkg, 5)
    (3.0 * loss).backward()
    assert abs(float(loss.detach()) - float(g["loss"])) <= LOSS_RTOL * abs(float(g["loss"]))
    gd, gn = d.grad.cpu().numpy() / 3.0, n.grad.cpu().numpy() / 3.0
    assert np.abs(gd - g["grad_depth"]).max() <= GRAD_TOL * np.abs(g["grad_depth"]).max()
    assert np.abs(gn - g["grad_normal"]).max() <= GRAD_TOL * np.abs(g["grad_normal"]).max()


def _view(W, H, seed):
    """A camera of the given size looking at the cases' sphere, with its planes."""
    cam = S.ring_cameras(1, 2.2, W, H, fovx_deg=55.0, phase=0.3 + seed)[0]
    return (cam,) + nd_inputs(dict(W=W, H=H, seed=seed), cam.c2w, cam=cam)


@pytest.mark.parametrize("mode,ks,tol_deg", [("dmean", 3, 90.0), ("dmean", 7, 75.0), ("dmed", 3, None)])
def test_packed_views_match_oracle(mode, ks, tol_deg):
    """Three views of different sizes, one of them 800x800, packed as the render packs them."""
    from oracle import oracle as O
    per = [_view(800, 800, 3), _view(173, 91, 5), _view(64, 200, 7)]
    cams = [p[0] for p in per]
    depth = torch.from_numpy(np.concatenate([p[1].reshape(-1) for p in per])).cuda()
    normal = torch.from_numpy(np.concatenate([p[2].reshape(-1) for p in per])).cuda()
    T = torch.from_numpy(np.concatenate([p[3].reshape(-1) for p in per])).cuda()
    tol = float(np.float32(np.cos(np.deg2rad(tol_deg)))) if tol_deg else -1.0
    loss, gd, gn = LU.normal_depth_loss_views(cams, depth, normal, T, mode, ks, tol, weight=0.5)
    loss, gd, gn = loss.cpu().numpy(), gd.cpu().numpy(), gn.cpu().numpy()
    plane = 0 if mode == "dmean" else 2
    off = 0
    for i, (cam, d, n, t) in enumerate(per):
        HW = cam.width * cam.height
        ref = O.normal_depth_loss(cam.width, cam.height, cam.cx, cam.cy, cam.tanfovx, cam.tanfovy, cam.c2w, d[plane],
                                  n, t[0] if mode == "dmean" else None, ks, tol)
        assert abs(loss[i] - 0.5 * ref[0]) <= LOSS_RTOL * abs(0.5 * ref[0])
        gdv = gd[4 * off:4 * (off + HW)].reshape(4, cam.height, cam.width)
        gnv = gn[3 * off:3 * (off + HW)].reshape(3, cam.height, cam.width)
        assert np.abs(gdv[plane] - 0.5 * ref[1]).max() <= GRAD_TOL * 0.5 * np.abs(ref[1]).max()
        assert not np.delete(gdv, plane, axis=0).any()
        assert np.abs(gnv - 0.5 * ref[2]).max() <= GRAD_TOL * 0.5 * np.abs(ref[2]).max()
        off += HW


def test_gradients_accumulate_and_small_images():
    cam, d, n, t = _view(96, 64, 9)
    depth, normal, T = (torch.from_numpy(a.reshape(-1)).cuda() for a in (d, n, t))
    l1, gd1, gn1 = LU.normal_depth_loss_views([cam], depth, normal, T, "dmean", 3, -1.0)
    l2, gd2, gn2 = LU.normal_depth_loss_views([cam], depth, normal, T, "dmean", 3, -1.0, grad_depth=gd1.clone(),
                                              grad_normal=gn1.clone(), loss_out=l1.clone())
    assert torch.allclose(gd2, 2 * gd1) and torch.allclose(gn2, 2 * gn1) and torch.allclose(l2, 2 * l1)
    # no interior pixel for a 9-wide stencil on a 6x5 image: zero loss, zero gradients
    tiny = S.ring_cameras(1, 2.2, 6, 5, fovx_deg=55.0)[0]
    z = LU.normal_depth_loss_views([tiny], torch.ones(4 * 30, device="cuda"), torch.ones(3 * 30, device="cuda"),
                                   torch.zeros(30, device="cuda"), "dmean", 9, -1.0)
    assert float(z[0]) == 0.0 and not z[1].any() and not z[2].any()
    with pytest.raises(RuntimeError):
        LU.normal_depth_loss_views([cam], depth, normal, T, "dmean", 4, -1.0)


def test_training_step_adds_the_losses_to_the_upstream_planes():
    """BatchedTrainStep(normal_losses=...): the planes the adjoint reads are the seeded upstream
    gradients plus both losses' gradients on that step's rendered planes; a graph replay of the
    step computes the same losses as the eager step on the same parameters."""
    from svraster_b200.step import BatchedTrainStep
    sc = S.scene_small(seed=2)
    cams = S.fibonacci_cameras(3, 3.0, 144, 112, fovx_deg=50.0)
    nl = dict(lambda_dmean=0.5, dmean_ks=3, dmean_tol_deg=90.0, lambda_dmed=0.25)
    a = BatchedTrainStep(sc, cams, device="cuda", lambda_R_concen=0.1, normal_losses=nl)
    b = BatchedTrainStep(sc, cams, device="cuda", lambda_R_concen=0.1, normal_losses=nl)
    b.capture()
    a.step()
    b.replay()
    torch.cuda.synchronize()
    st = a.state
    _, depth, normal, T, _ = st.render(3, True, True, a.centers, a.lengths, a.geos, a.rgbs, a.s_val,
                                       rgb_per_view=True)
    tol = float(np.float32(np.cos(np.deg2rad(90.0))))
    l0, gd, gn = LU.normal_depth_loss_views(a.views, depth, normal, T, "dmean", 3, tol, 0.5)
    l1, gd, gn = LU.normal_depth_loss_views(a.views, depth, normal, T, "dmed", 3, -1.0, 0.25, gd, gn, l0)
    assert float(l1.sum()) > 0
    torch.testing.assert_close(a.nd_loss, l1, rtol=1e-9, atol=0)
    torch.testing.assert_close(a.ddepth_w - a.ddepth, gd, rtol=0, atol=1e-6)
    torch.testing.assert_close(a.dnormal_w - a.dnormal, gn, rtol=0, atol=1e-6)
    # the replay rendered from the same initial parameters: the same losses to float rounding
    torch.testing.assert_close(b.nd_loss, a.nd_loss, rtol=1e-6, atol=0)
    assert b.graph_status() == (0, 0)
