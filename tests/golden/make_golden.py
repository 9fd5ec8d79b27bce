"""Generate golden vectors from the reference's own CUDA extension (run on a B200).

The reference extension is built from its unmodified sources into ``oracle/_ref`` by
``oracle/build_ref.py`` (which also builds its smoothness adjoints once more with the
clock64() seed fixed by a compile prelude).  This script runs the reference ops on seeded
synthetic inputs and writes ``<out>/<case>.npz`` with the outputs; inputs are regenerated
by the tests from the same seeds and checked against the stored input digest.

The reference backward reads the depth and normal gradient planes unconditionally
(backward.cu:180-184), so every case renders with need_depth and need_normal on.

Usage (GPU machine):  python tests/golden/make_golden.py [--out DIR] [--only reg ...]
(default DIR: tests/golden/_new; the fixtures that pass review are copied into tests/golden/)
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests.golden.cases import CASES, TABLE_CASE, ADAM_CASE, REG_CASE, build_case_inputs, build_table_inputs, \
    build_adam_inputs, build_reg_inputs, digest  # noqa: E402


def load_module(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def chunk_offsets(base_ptr, sizes_aligns):
    """Offsets of RASTER_STATE::obtain partitions (cuda/src/raster_state.cu:37-43)."""
    offs, p = [], base_ptr
    for size, align in sizes_aligns:
        p = (p + align - 1) & ~(align - 1)
        offs.append(p - base_ptr)
        p += size
    return offs


def unpack_geom(buf, P):
    off = chunk_offsets(buf.data_ptr(), [(4 * P, 128), (4 * P, 128), (8 * P, 128), (4 * P, 128)])
    b = buf.cpu().numpy()
    ndup = b[off[0]:off[0] + 4 * P].view(np.uint32)
    bbox = b[off[2]:off[2] + 8 * P].view(np.uint32).reshape(P, 2)
    bits = b[off[3]:off[3] + 4 * P].view(np.uint32)
    return ndup.copy(), bbox.copy(), bits.copy()


def unpack_binning(buf, R):
    off = chunk_offsets(buf.data_ptr(), [(8 * R, 128), (8 * R, 128), (4 * R, 128), (4 * R, 128)])
    b = buf.cpu().numpy()
    keys = b[off[1]:off[1] + 8 * R].view(np.uint64)
    vals = b[off[3]:off[3] + 4 * R].view(np.uint32)
    return keys.copy(), vals.copy()


def unpack_image(buf, HW, T):
    off = chunk_offsets(buf.data_ptr(), [(8 * T, 128), (4 * T, 128), (4 * HW, 128)])
    b = buf.cpu().numpy()
    ranges = b[off[0]:off[0] + 8 * T].view(np.uint32).reshape(T, 2)
    tl = b[off[1]:off[1] + 4 * T].view(np.uint32)
    nc = b[off[2]:off[2] + 4 * HW].view(np.uint32)
    return ranges.copy(), tl.copy(), nc.copy()


def run_render_case(R_, case, dev):
    inp = build_case_inputs(case)
    sc, cam, grads = inp["scene"], inp["cam"], inp["grads"]
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    octpath = t(sc.octpath, torch.int64)
    centers, lengths = t(sc.vox_center), t(sc.vox_size)
    is_leaf = t(sc.is_leaf, torch.uint8)
    w2c, c2w = t(cam.w2c), t(cam.c2w)
    bg = t(np.asarray(case["bg"], np.float32))
    W, H = cam.width, cam.height
    ndup_t, geom = R_.rasterize_preprocess(W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0, cam.near,
                                           octpath, centers, lengths, is_leaf, False)
    care = torch.where(ndup_t > 0)[0]
    vox_key = t(sc.vox_key, torch.int64)
    grid = t(sc.geo_grid_pts)
    geos = R_.gather_triinterp_geo_params(vox_key, care, grid)
    rgbs = R_.sh_compute(3, care, centers, c2w[:3, 3].contiguous(), t(sc.sh0), t(sc.shs))
    s_val = torch.exp(torch.tensor([sc.log_s], dtype=torch.float32, device=dev) * 10.0)
    out = R_.rasterize_voxels(case["vox_geo_mode"], 1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w,
                              bg, 0, True, False, True, True, octpath, centers, lengths, geos, rgbs,
                              torch.empty(sc.n_vox, 0, device=dev), geom, False, s_val)
    num_rendered, binning, imgbuf, color, depth, normal, T, max_w = out[:8]
    lam = case["lambda_R_concen"]
    gt = t(grads["gt"])
    bw = R_.rasterize_voxels_backward(num_rendered, 3, 1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w,
                                      bg, octpath, centers, lengths, geos, rgbs, geom, binning, imgbuf, T,
                                      t(grads["color"]), t(grads["depth"]), t(grads["normal"]), t(grads["T"]),
                                      lam, gt, 0.0, 0.0, True, True, depth, normal, False, s_val, out[8])
    dgeos, drgbs, dsub, ds = bw
    dgrid = R_.gather_triinterp_geo_params_bw(vox_key, care, grid.numel(), dgeos.contiguous())
    dsh0, dshs = R_.sh_compute_bw(3, 16, care, centers, c2w[:3, 3].contiguous(), rgbs, drgbs.contiguous())
    torch.cuda.synchronize()
    N = sc.n_vox
    ndup, bbox, bits = unpack_geom(geom, N)
    keys, vals = unpack_binning(binning, num_rendered)
    T_t = ((W + 15) // 16) * ((H + 15) // 16)
    ranges, tl, nc = unpack_image(imgbuf, W * H, T_t)
    care_np = care.cpu().numpy()
    dvox = torch.cat([dgeos, drgbs, dsub], 1).cpu().numpy()
    rows = np.where(np.abs(dvox).sum(1) > 0)[0]
    g = lambda x: x.detach().cpu().numpy()
    return dict(digest=digest(inp), n_dup=g(ndup_t), geom_ndup=ndup, bbox=bbox, bits=bits, num_rendered=num_rendered,
                keys=keys, vals=vals, ranges=ranges, tile_last=tl, n_contrib=nc, care=care_np,
                geos=g(geos)[care_np], rgbs=g(rgbs)[care_np], color=g(color), depth=g(depth), normal=g(normal),
                T=g(T), max_w=g(max_w), dvox_rows=rows, dvox=dvox[rows], ds=g(ds), dgrid=g(dgrid).reshape(-1),
                dsh0=g(dsh0)[care_np], dshs=g(dshs)[care_np])


def run_table_case(R_, S_, case, dev):
    inp = build_table_inputs(case)
    sc = inp["scene"]
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    centers, sizes = t(sc.vox_center), t(sc.vox_size)
    leaf = t(sc.is_leaf.astype(bool), torch.bool)
    sc_center = t(np.zeros(3, np.float32))
    res_pow2 = case["res_pow2"]
    N = sc.n_vox
    if inp["expected_count"] > N * 64:
        raise RuntimeError("table case would overflow the reference's N*64 slot buffer")
    mask, keys, g2v = R_.valid_gradient_table(centers, sizes, sc_center, float(sc.scene_extent), res_pow2, leaf)
    order = torch.argsort(keys.to(torch.int64) * (N + 1) + g2v.to(torch.int64))
    keys, g2v = keys[order].contiguous(), g2v[order].contiguous()
    res = 1 << res_pow2
    coord, vsize = t(inp["grid_voxel_coord"]), t(inp["grid_voxel_size"])
    active = t(inp["active"], torch.int32)
    grid = t(sc.geo_grid_pts)
    vox_key = t(sc.vox_key, torch.int64)
    out = dict(digest=digest(inp), mask=mask.cpu().numpy(), keys=keys.cpu().numpy(), g2v=g2v.cpu().numpy())
    for name, fn in (("lap", S_.laplacian_smoothness_bw), ("eik", S_.grid_eikonal_bw)):
        gg = torch.zeros_like(grid)
        fn(grid, vox_key, coord, vsize, res, mask, keys, g2v, active, case["weight"], case["vox_size_inv"], True,
           False, gg)
        torch.cuda.synchronize()
        out[name] = gg.cpu().numpy().reshape(-1)
    out["seed"] = np.int64(S_.SEED)
    return out


def run_adam_case(R_, case, dev):
    inp = build_adam_inputs(case)
    out = dict(digest=digest(inp))
    for biased in (False, True):
        for sparse in (False, True):
            p = torch.as_tensor(inp["param"]).to(dev).clone()
            g = torch.as_tensor(inp["grad"]).to(dev)
            m = torch.as_tensor(inp["m"]).to(dev).clone()
            v = torch.as_tensor(inp["v"]).to(dev).clone()
            if biased:
                R_.biased_adam_step(sparse, p, g, m, v, case["lr"], case["beta1"], case["beta2"], case["eps"])
            else:
                R_.unbiased_adam_step(sparse, p, g, m, v, case["step"], case["lr"], case["beta1"], case["beta2"],
                                      case["eps"])
            torch.cuda.synchronize()
            k = f"{'b' if biased else 'u'}{'s' if sparse else 'd'}"
            out[k + "_p"], out[k + "_m"], out[k + "_v"] = p.cpu().numpy(), m.cpu().numpy(), v.cpu().numpy()
    return out


def run_reg_case(R_, case, dev):
    inp = build_reg_inputs(case)
    sc = inp["scene"]
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    w = case["weight"]
    grid1, grid3, vox_key = t(sc.geo_grid_pts), t(inp["grid3"]), t(sc.vox_key, torch.int64)
    vsi = t(inp["vox_size_inv"])
    out = dict(digest=digest(inp))
    g = t(inp["grad1"])
    R_.voxel_gradient_bw(grid1, vox_key, vsi, t(inp["active"], torch.int32), w, False, False, g)
    torch.cuda.synchronize()
    out["vg"] = g.cpu().numpy()
    for no_tv_s in (False, True):
        for name, grid, g0 in (("1", grid1, inp["grad1"]), ("3", grid3, inp["grad3"])):
            g = t(g0)
            R_.total_variation_bw(grid, vox_key, w, vsi, no_tv_s, False, g)
            torch.cuda.synchronize()
            out[f"tv{name}_{int(no_tv_s)}"] = g.cpu().numpy()
    tb = inp["table"]
    g = t(inp["grad1"])
    R_.points_loss_bw(t(inp["points"]), grid1, vox_key, t(inp["grid_voxel_coord"]), t(inp["grid_voxel_size"]),
                      1 << case["res_pow2"], t(tb["mask"], torch.bool), t(tb["keys"], torch.int32),
                      t(tb["g2v"], torch.int32), w, 1.0, True, False, g)
    torch.cuda.synchronize()
    out["pl"] = g.cpu().numpy()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "_new"))
    ap.add_argument("--only", nargs="*", default=None,
                    help="fixtures to (re)write, e.g. reg table; default all")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    dev = torch.device("cuda:0")
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    R_ = load_module(os.path.join(ref_dir, "svraster_ref_C.so"), "svraster_ref_C")
    S_ = load_module(os.path.join(ref_dir, "seeded", "svraster_ref_seeded_C.so"), "svraster_ref_seeded_C")
    want = lambda n: args.only is None or n in args.only
    save = lambda n, res: np.savez_compressed(os.path.join(args.out, f"{n}.npz"), **res)
    for name, case in CASES.items():
        if want(name):
            res = run_render_case(R_, case, dev)
            save(name, res)
            print(name, "R =", res["num_rendered"])
    if want("table"):
        res = run_table_case(R_, S_, TABLE_CASE, dev)
        save("table", res)
        print("table G =", len(res["keys"]))
    if want("adam"):
        save("adam", run_adam_case(R_, ADAM_CASE, dev))
    if want("reg"):
        save("reg", run_reg_case(R_, REG_CASE, dev))
    print("done")


if __name__ == "__main__":
    main()
