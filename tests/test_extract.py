"""TSDF fusion and sparse marching cubes: the CPU restatement (oracle/extract_oracle.py) and
the sm_100a library against golden vectors from the reference's own torch code."""
import os
import types

import numpy as np
import pytest
import torch

from tests.golden.extract_cases import MC_CASES, TSDF_CASES, mc_inputs, mesh_digest, tsdf_inputs

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(HERE, f"extract_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture extract_{name}.npz missing")
    return dict(np.load(path))


def _oracle_tsdf(case, inp, g):
    from oracle import extract_oracle as X
    M = len(inp["xyz"])
    w = np.zeros((M, 1), np.float32)
    s = np.zeros((M, 1), np.float32)
    for k, cam in enumerate(inp["cams"]):
        X.tsdf_integrate(w, s, inp["xyz"], g["w2c"][k], g["c2w"][k], g["tanfov"][k][0], g["tanfov"][k][1], 0.5, 0.5,
                         inp["depths"][k], inp["alphas"][k], inp["bandwidth"], use_trunc=case["use_trunc"],
                         alpha_thres=case["alpha_thres"], crop_border=case["crop_border"],
                         depth_weight=case["depth_weight"], border_weight=case["border_weight"])
    return w, s


def _compare_tsdf(w, s, g, tol):
    """Accumulators within tol (relative to max(1, |value|)); a grid point whose sample
    lands exactly on a filter threshold may flip, so a few are allowed to differ."""
    ref_w, ref_s = g["weight"], g["sd_val"]
    bad = (np.abs(w - ref_w) > tol * np.maximum(1, np.abs(ref_w))) | \
          (np.abs(s - ref_s) > tol * np.maximum(1, np.abs(ref_s)))
    assert bad.mean() <= 2e-3, f"{bad.sum()} of {bad.size} accumulators differ"
    fused = (ref_w[:, 0] > 0) & ~bad[:, 0]
    t = s[fused, 0] / w[fused, 0]
    ref_t = ref_s[fused, 0] / ref_w[fused, 0]
    np.testing.assert_allclose(t, ref_t, rtol=tol, atol=tol)


@pytest.mark.parametrize("name", list(TSDF_CASES))
def test_oracle_tsdf_matches_reference(name):
    g = load(name)
    case = TSDF_CASES[name]
    inp = tsdf_inputs(case)
    assert str(g["digest"]) == inp["digest"]
    w, s = _oracle_tsdf(case, inp, g)
    _compare_tsdf(w, s, g, 1e-5)


@pytest.mark.parametrize("name", list(MC_CASES))
def test_oracle_marching_cubes_matches_reference_bitexact(name):
    from oracle import extract_oracle as X
    g = load(name)
    inp = mc_inputs(MC_CASES[name])
    assert str(g["digest"]) == inp["digest"]
    v, f = X.marching_cubes(inp["val"], inp["xyz"], inp["vox_key"], MC_CASES[name]["iso"])
    _assert_mesh_equal(v, f, g)


def _assert_mesh_equal(v, f, g):
    """Bit-exact mesh: against the full arrays, or (compact fixtures) against the digests of
    their exact bytes, with counts and sampled rows checked first for a readable failure."""
    if "verts" in g:
        assert np.array_equal(v, g["verts"])
        assert np.array_equal(f, g["faces"])
        return
    assert (len(v), len(f)) == (int(g["n_verts"]), int(g["n_faces"]))
    assert np.array_equal(np.asarray(v, np.float32)[g["vert_rows"]], g["verts_sample"])
    assert np.array_equal(np.asarray(f, np.int64)[g["face_rows"]], g["faces_sample"])
    d = mesh_digest(v, f)
    assert d["verts_sha256"] == str(g["verts_sha256"]) and d["faces_sha256"] == str(g["faces_sha256"])


def _ref_cam(g, k, inp):
    c = inp["cams"][k]
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()
    return types.SimpleNamespace(w2c=t(g["w2c"][k]), c2w=t(g["c2w"][k]), tanfovx=float(g["tanfov"][k][0]),
                                 tanfovy=float(g["tanfov"][k][1]), cx_p=0.5, cy_p=0.5, image_width=c.width,
                                 image_height=c.height, near=0.02)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(TSDF_CASES))
def test_library_tsdf_matches_reference(name):
    from svraster_b200.fuser import Fuser
    g = load(name)
    case = TSDF_CASES[name]
    inp = tsdf_inputs(case)
    bw = inp["bandwidth"]
    bw = torch.as_tensor(bw).cuda() if isinstance(bw, np.ndarray) else bw
    kw = dict(use_trunc=case["use_trunc"], alpha_thres=case["alpha_thres"], crop_border=case["crop_border"],
              depth_weight=case["depth_weight"], border_weight=case["border_weight"])
    xyz = torch.as_tensor(inp["xyz"]).cuda()
    fz = Fuser(xyz, bw, **kw)
    for k in range(len(inp["cams"])):
        fz.integrate(_ref_cam(g, k, inp), torch.as_tensor(inp["depths"][k]).cuda(),
                     alpha=torch.as_tensor(inp["alphas"][k]).cuda())
    w, s = fz.weight.cpu().numpy(), fz.sd_val.cpu().numpy()
    _compare_tsdf(w, s, g, 1e-5)
    # one batched launch over all views gives the same float32 accumulators
    fb = Fuser(xyz, bw, **kw)
    fb.integrate_batch([_ref_cam(g, k, inp) for k in range(len(inp["cams"]))],
                       [torch.as_tensor(d).cuda() for d in inp["depths"]],
                       [torch.as_tensor(a).cuda() for a in inp["alphas"]])
    assert np.array_equal(fb.weight.cpu().numpy(), w)
    assert np.array_equal(fb.sd_val.cpu().numpy(), s)
    # float64 accumulators: same fused set, close values
    f64 = Fuser(xyz, bw, precision="fp64", **kw)
    f64.integrate_batch([_ref_cam(g, k, inp) for k in range(len(inp["cams"]))],
                        [torch.as_tensor(d).cuda() for d in inp["depths"]],
                        [torch.as_tensor(a).cuda() for a in inp["alphas"]])
    np.testing.assert_allclose(f64.weight.cpu().numpy(), w, rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(MC_CASES))
def test_library_marching_cubes_matches_reference_bitexact(name):
    from svraster_b200.marching_cubes import torch_marching_cubes_grid
    g = load(name)
    inp = mc_inputs(MC_CASES[name])
    v, f = torch_marching_cubes_grid(torch.as_tensor(inp["val"]).cuda(), torch.as_tensor(inp["xyz"]).cuda(),
                                     torch.as_tensor(inp["vox_key"]).cuda(), MC_CASES[name]["iso"])
    _assert_mesh_equal(v.cpu().numpy(), f.cpu().numpy(), g)


@pytest.mark.gpu
def test_marching_cubes_properties_mid_scene():
    """At the benchmark scene's size: sorted unique vertices, valid non-degenerate faces and
    the fp64 interpolation mode within float rounding of the fp32 one."""
    from svraster_b200 import synthetic as S
    from svraster_b200.marching_cubes import torch_marching_cubes_grid
    sc = S.scene_mid()
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    v, f = torch_marching_cubes_grid(t(sc.geo_grid_pts), t(sc.grid_pts_xyz), t(sc.vox_key), 0.0)
    vv, ff = v.cpu().numpy(), f.cpu().numpy()
    assert len(ff) > 100000
    assert ff.min() >= 0 and ff.max() < len(vv)
    d = np.diff(vv.view(np.uint32).astype(np.int64), axis=0)
    order = np.lexsort(vv.T[::-1])
    assert np.array_equal(order, np.arange(len(vv))), "vertices not lexicographically sorted"
    assert len(np.unique(vv, axis=0)) == len(vv)
    v64, f64 = torch_marching_cubes_grid(t(sc.geo_grid_pts), t(sc.grid_pts_xyz), t(sc.vox_key), 0.0, fp64=True)
    assert len(f64) == len(f)
