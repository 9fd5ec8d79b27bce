"""The drop-in Python surface end to end: svraster_cuda.renderer.rasterize_voxels with the
model's vox_fn (GatherGeoParams + SH_eval) and torch autograd, against the C oracle chain
(render adjoint -> gather adjoint / SH adjoint) on the same inputs."""
import numpy as np
import pytest
import torch

from svraster_b200 import synthetic as S
from tests.helpers import oracle_inputs, oracle_view, upstream_grads

pytestmark = pytest.mark.gpu


def test_install_as_svraster_cuda():
    import svraster_b200
    svraster_b200.install_as_svraster_cuda()
    import svraster_cuda
    from svraster_cuda import renderer
    assert svraster_cuda is svraster_b200 and renderer is svraster_b200.renderer
    assert svraster_cuda.meta.MAX_NUM_LEVELS == 16


def _settings(renderer, cam, dev, **kw):
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).to(dev)
    base = dict(color_mode="sh", vox_geo_mode="triinterp3", density_mode="sdf", image_width=cam.width,
                image_height=cam.height, tanfovx=cam.tanfovx, tanfovy=cam.tanfovy, cx=cam.cx, cy=cam.cy,
                w2c_matrix=t(cam.w2c), c2w_matrix=t(cam.c2w), background=torch.zeros(3, device=dev), near=cam.near,
                need_depth=True, need_normal=True)
    base.update(kw)
    return renderer.RasterSettings(**base)


def test_rasterize_voxels_autograd_matches_oracle_chain():
    from oracle import oracle as O
    from svraster_b200 import renderer
    dev = torch.device("cuda")
    sc = S.scene_small(seed=4)
    cam = S.ring_cameras(1, 3.0, 128, 96, phase=1.1)[0]
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    grid = t(sc.geo_grid_pts).requires_grad_(True)
    sh0 = t(sc.sh0).requires_grad_(True)
    shs = t(sc.shs).requires_grad_(True)
    log_s = torch.tensor([sc.log_s], dtype=torch.float32, device=dev).requires_grad_(True)
    vox_key, centers, lengths = t(sc.vox_key, torch.int64), t(sc.vox_center), t(sc.vox_size)

    def vox_fn(idx, cam_pos, color_mode):
        geos = renderer.GatherGeoParams.apply("triinterp3", vox_key, 1.0 / lengths, idx, grid)
        rgbs = renderer.SH_eval.apply(3, idx, centers, cam_pos, None, sh0, shs)
        return dict(geos=geos, rgbs=rgbs, subdiv_p=torch.zeros(sc.n_vox, 1, device=dev), log_s=log_s)

    g = upstream_grads(cam.height, cam.width, seed=9)[0]
    rs = _settings(renderer, cam, dev, lambda_R_concen=0.1, gt_color=t(g["gt"]))
    color, depth, normal, T, max_w, feat = renderer.rasterize_voxels(rs, t(sc.octpath, torch.int64), centers,
                                                                     lengths, vox_fn, t(sc.is_leaf, torch.uint8))
    assert color.shape == (3, cam.height, cam.width) and depth.shape == (4, cam.height, cam.width)
    assert normal.shape == (3, cam.height, cam.width) and T.shape == (1, cam.height, cam.width)
    assert feat.shape == (0, cam.height, cam.width)
    torch.autograd.backward([color, depth, normal, T], [t(g["color"]), t(g["depth"]), t(g["normal"]), t(g["T"])])

    geos_o, rgbs_o = oracle_inputs(sc, cam)
    ref = oracle_view(sc, cam, geos_o, rgbs_o, grads=g, lambda_R=0.1)
    np.testing.assert_allclose(color.detach().cpu().numpy(), ref["color"], rtol=1e-4, atol=1e-4)
    vis = np.where(ref["n_dup"] > 0)[0]
    dgrid = O.gather_geo_bw(vis, sc.vox_key, ref["dvox"][:, :8], len(sc.geo_grid_pts))
    dsh0, dshs = O.sh_eval_bw(3, vis, sc.vox_center, cam.position, ref["dvox"][:, 8:11], 16)
    for name, got, exp in (("grid", grid.grad, dgrid), ("sh0", sh0.grad, dsh0), ("shs", shs.grad, dshs)):
        got = got.detach().cpu().numpy().reshape(exp.shape)
        scale = np.abs(exp).max() + 1e-12
        assert np.quantile(np.abs(got - exp) / scale, 0.999) < 1e-3, name
    # s = exp(10 log_s): dL/dlog_s = dL/ds * 10 s
    exp_ls = ref["ds"] * 10.0 * sc.s_val
    assert abs(log_s.grad.item() - exp_ls) <= 1e-3 * abs(exp_ls) + 1e-3


def test_unsupported_modes_raise():
    from svraster_b200 import renderer
    dev = torch.device("cuda")
    sc = S.scene_tiny()
    cam = S.ring_cameras(1, 3.0, 32, 32)[0]
    for kw in (dict(density_mode="exp_linear_11"), dict(cam_mode="ortho"), dict(lambda_dist=0.1)):
        rs = _settings(renderer, cam, dev, **kw)
        with pytest.raises(NotImplementedError):
            renderer.rasterize_voxels(rs, torch.zeros(4, dtype=torch.int64, device=dev),
                                      torch.zeros(4, 3, device=dev), torch.ones(4, 1, device=dev), None,
                                      torch.ones(4, dtype=torch.uint8, device=dev))
