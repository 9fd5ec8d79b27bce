"""Time the reference's own CUDA extension (oracle/_ref, built from its unmodified sources) on
the benchmark workload, one view at a time as the reference trains -- TEST INFRASTRUCTURE.

Per view: rasterize_preprocess, gather + SH (care = in-frustum voxels), rasterize_voxels,
rasterize_voxels_backward, gather / SH adjoints.  Per step (8 views): the Laplacian and
grid-Eikonal adjoints over every dense-grid key and Adam on grid / sh0 / shs, i.e. the same
work as one batched step of svraster_b200.step.BatchedTrainStep.  CUDA events, median of
the timed steps.  Prints one JSON line.

Usage (GPU machine):  python oracle/time_reference_gpu.py [--steps 5 --warmup 2] [--regularisers]
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def load_module(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def time_checkpoint_oracle(args):
    """The reference builds the checkpoint codebook with torch ops (io.py:123-167), which do not
    exist outside its Python tree; its CPU behaviour is restated bit for bit by the C oracle,
    timed here single-threaded on the same 19 tensors bench.run_checkpoint codes."""
    import time
    import bench
    # this script's own folder is first on sys.path, so load the oracle front-end by path
    O = load_module(os.path.join(ROOT, "oracle", "oracle.py"), "svr_oracle_front")
    scene, _ = bench.make_workload(0, config=args.config)
    cols = [scene.geo_grid_pts.reshape(-1)] + [scene.sh0[:, j] for j in range(scene.sh0.shape[1])] + \
        [scene.shs[:, j] for j in range(scene.shs.shape[1])]
    t0 = time.perf_counter()
    for c in cols:
        O.quantize(np.ascontiguousarray(c, dtype=np.float32))
    ms = (time.perf_counter() - t0) * 1e3
    print(json.dumps({"impl": "C oracle (restates io.py:123-167), 1 thread", "workload": "checkpoint",
                      "values": int(sum(c.size for c in cols)), "codebooks": len(cols),
                      "quantize_ms": round(ms, 1), "cores": 1}), flush=True)


def time_regularisers(R_, bench, scene, grid, vox_key, mask, keys, g2v, coord, vsize, res, dev):
    """The reference's voxel_gradient_bw, total_variation_bw (dense, tv_sparse) and
    points_loss_bw on the inputs bench.run_regularisers times, timed the same way: CUDA events
    around 10 back-to-back calls, median of 5."""
    active, vsi, pts = bench.regulariser_inputs(scene, mask, res, dev)
    grad = torch.zeros_like(grid)

    def timed(fn, calls=10, reps=5):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(calls):
                fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) / calls)
        return round(float(np.median(ts)), 4)

    out = {"impl": "reference CUDA extension", "workload": "regularisers", "voxels": scene.n_vox,
           "grid_points": int(grid.shape[0]), "points": int(pts.shape[0]),
           "voxel_gradient_ms": timed(lambda: R_.voxel_gradient_bw(grid, vox_key, vsi, active, 1e-3, False, False,
                                                                   grad)),
           "total_variation_ms": timed(lambda: R_.total_variation_bw(grid, vox_key, 1e-3, vsi, False, False, grad)),
           "total_variation_sparse_ms": timed(lambda: R_.total_variation_bw(grid, vox_key, 1e-3, vsi, False, True,
                                                                            grad)),
           "points_loss_ms": timed(lambda: R_.points_loss_bw(pts, grid, vox_key, coord, vsize, res, mask, keys, g2v,
                                                             1e-3, 1.0, True, False, grad))}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--config", default="mid", help="bench.py workload (mid | batched)")
    ap.add_argument("--regularisers", action="store_true",
                    help="time voxel_gradient_bw / total_variation_bw / points_loss_bw instead of the step")
    ap.add_argument("--checkpoint", action="store_true",
                    help="time the C oracle's 8-bit checkpoint codebook on the bench model instead")
    args = ap.parse_args()
    if args.checkpoint:
        time_checkpoint_oracle(args)
        return
    import bench
    R_ = load_module(os.path.join(ROOT, "oracle", "_ref", "svraster_ref_C.so"), "svraster_ref_C")
    dev = torch.device("cuda:0")
    scene, cams = bench.make_workload(0, config=args.config)
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    octpath, centers, lengths = t(scene.octpath, torch.int64), t(scene.vox_center), t(scene.vox_size)
    is_leaf = t(scene.is_leaf, torch.uint8)
    vox_key, grid = t(scene.vox_key, torch.int64), t(scene.geo_grid_pts)
    sh0, shs = t(scene.sh0), t(scene.shs)
    s_val = torch.exp(torch.tensor([scene.log_s], dtype=torch.float32, device=dev) * 10.0)
    views = [(t(c.w2c), t(c.c2w), c) for c in cams]
    bg = torch.zeros(3, device=dev)
    g = torch.Generator(device=dev).manual_seed(0)
    P = cams[0].width * cams[0].height
    ups = [(torch.randn(3, c.height, c.width, device=dev, generator=g),
            torch.randn(4, c.height, c.width, device=dev, generator=g),
            torch.randn(3, c.height, c.width, device=dev, generator=g),
            torch.zeros(1, c.height, c.width, device=dev),
            torch.rand(3, c.height, c.width, device=dev, generator=g)) for c in cams]
    res_pow2 = min(int(scene.octlevel.max()), 9)
    res = 1 << res_pow2
    mask, keys, g2v = R_.valid_gradient_table(centers, lengths, torch.zeros(3, device=dev),
                                              float(scene.scene_extent), res_pow2, is_leaf.bool())
    order = torch.argsort(keys)
    keys, g2v = keys[order].contiguous(), g2v[order].contiguous()
    ext = np.float32(scene.scene_extent)
    coord = t(np.round(((scene.vox_center - scene.vox_size * np.float32(0.5)) + ext * np.float32(0.5)) / ext
                       * np.float32(res)))
    vsize = t(np.round(scene.vox_size / ext * np.float32(res))).reshape(-1)
    active = torch.arange(keys.numel(), dtype=torch.int32, device=dev)
    if args.regularisers:
        time_regularisers(R_, bench, scene, grid, vox_key, mask, keys, g2v, coord, vsize, res, dev)
        return
    params = [grid, sh0, shs]
    ms_ = [torch.zeros_like(p) for p in params]
    vs_ = [torch.zeros_like(p) for p in params]

    stage = {"preprocess": 0.0, "render_fwd": 0.0, "render_bwd": 0.0}

    def one_step(it, timed):
        dgrid = torch.zeros_like(grid)
        dsh0 = torch.zeros_like(sh0)
        dshs = torch.zeros_like(shs)
        for (w2c, c2w, c), (dc, dd, dn, dT, gt) in zip(views, ups):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
            e[0].record()
            ndup, geom = R_.rasterize_preprocess(c.width, c.height, c.tanfovx, c.tanfovy, c.cx, c.cy, w2c, c2w, 0,
                                                 c.near, octpath, centers, lengths, is_leaf, False)
            e[1].record()
            care = torch.where(ndup > 0)[0]
            geos = R_.gather_triinterp_geo_params(vox_key, care, grid)
            cam_pos = c2w[:3, 3].contiguous()
            rgbs = R_.sh_compute(3, care, centers, cam_pos, sh0, shs)
            e[2].record()
            out = R_.rasterize_voxels(3, 1, c.width, c.height, c.tanfovx, c.tanfovy, c.cx, c.cy, w2c, c2w, bg, 0,
                                      True, False, True, False, octpath, centers, lengths, geos, rgbs,
                                      torch.empty(scene.n_vox, 0, device=dev), geom, False, s_val)
            e[3].record()
            nr, binning, img, color, depth, normal, T = out[:7]
            e[4].record()
            dgeos, drgbs, _, ds = R_.rasterize_voxels_backward(
                nr, 3, 1, c.width, c.height, c.tanfovx, c.tanfovy, c.cx, c.cy, w2c, c2w, bg, octpath, centers,
                lengths, geos, rgbs, geom, binning, img, T, dc, dd, dn, dT, 0.1, gt, 0.0, 0.0, True, True, depth,
                normal, False, s_val, out[8])
            e[5].record()
            dgrid += R_.gather_triinterp_geo_params_bw(vox_key, care, grid.numel(), dgeos.contiguous())
            a0, a1 = R_.sh_compute_bw(3, 16, care, centers, cam_pos, rgbs, drgbs.contiguous())
            dsh0 += a0
            dshs += a1
            if timed:
                torch.cuda.synchronize()
                stage["preprocess"] += e[0].elapsed_time(e[1])
                stage["render_fwd"] += e[2].elapsed_time(e[3])
                stage["render_bwd"] += e[4].elapsed_time(e[5])
        R_.laplacian_smoothness_bw(grid, vox_key, coord, vsize, res, mask, keys, g2v, active, 1e-3,
                                   float(res) / scene.scene_extent, True, False, dgrid)
        R_.grid_eikonal_bw(grid, vox_key, coord, vsize, res, mask, keys, g2v, active, 1e-3,
                           float(res) / scene.scene_extent, True, False, dgrid)
        for p, gr, m, v, lr in zip(params, (dgrid, dsh0, dshs), ms_, vs_, (1e-3, 1e-3, 1e-4)):
            R_.unbiased_adam_step(False, p, gr, m, v, it + 1, lr, 0.1, 0.99, 1e-15)

    for i in range(args.warmup):
        one_step(i, False)
    torch.cuda.synchronize()
    times = []
    for i in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        one_step(args.warmup + i, True)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    rays = sum(c.width * c.height for c in cams)
    print(json.dumps({"impl": "reference CUDA extension (per view, default stream)", "workload": bench.CONFIGS[args.config]["workload"],
                      "ms_per_step": round(ms, 3), "Mrays_per_s": round(rays / ms / 1e3, 3),
                      "stage_ms_per_step": {k: round(v / args.steps, 3) for k, v in stage.items()},
                      "grid_keys": int(keys.numel())}), flush=True)


if __name__ == "__main__":
    main()
