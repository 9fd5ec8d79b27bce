"""Throughput benchmark of the sm_100a sparse-voxel SDF rasterizer training step.

Headline workload (batched): a sphere with 64 Gaussian bumps, octree levels 7-11 (~4.2M
voxels), SH degree 3, 64 views of mixed resolution (16 each of 480x360, 960x540, 1280x720,
1920x1080, shuffled; 58.9M rays) in one step: gather, SH, preprocess, binning (sort
included), render forward and adjoint, smoothness adjoints and Adam, captured as one CUDA
graph (svraster_b200.step).  ``--config mid`` is the plain mid-size workload (3 spheres and a
torus, levels 6-10, 8 views of 800x800); the default line carries it as ``mid_size``.

  value : forward+backward Mrays/s of the batched step, inputs resident in HBM
  per_view : the same work through the plain per-view kernels (the drop-in API one view at
          a time, as the reference's train.py drives it), same device-resident inputs
  e2e   : the batched step through the C-ABI training step (two CUDA graphs) with each
          step's upstream gradient planes and target image copied from pinned host memory
          and the mean transmittance read back; ``e2e_per_view`` is the same through the
          per-view API
  native_step : the same step issued and graph-captured by the library's own host code
          (svr_step_*, the C entry a host without Python uses), inputs resident in HBM
  reference_cuda : the reference's own CUDA extension (built from its unmodified sources)
          on the same views, per view, timed after our timed regions (a baseline leg)
  roofline : the dominant kernel's algorithmic bytes / CUDA-event duration vs the measured
          HBM copy bandwidth (MEASURED_PEAKS.json), and its FP32 / MUFU issue ceiling from
          measured pair counts (``compute``)
  cpu_baseline : the CPU oracle (single thread) on a sample of the same workload

``--impl reference`` times the CPU restatement of the reference algorithm (the reference's
only implementation of this path is CUDA) with all host threads on a bounded sample.
Multi-GPU (torchrun): every rank renders its own views (weak scaling) and the gradients are
all-reduced over NCCL before Adam.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # the headline: one step over 64 views of four resolutions
    "batched": dict(workload="batched: sphere with 64 bumps, levels 7-11, SH deg 3, 64 views (16 each of "
                             "480x360, 960x540, 1280x720, 1920x1080, shuffled)", views=64, image="mixed"),
    # plain method, mid-size scene
    "mid": dict(workload="mid-size: 3 spheres + torus, levels 6-10, SH deg 3, 8 views 800x800", views=8,
                image="800x800"),
    # full reconstruction step: room scene, 128 training views, TSDF of 200 maps, MC at level 12
    "full": dict(workload="full reconstruction: 4x3x2.5 room + 20 boxes/spheres, levels 8-12, SH deg 3, "
                          "128 views 1024x768; TSDF of 200 depth maps 1024x768 (trunc 3 voxels), MC at level 12",
                 views=128, image="1024x768"),
}
DEFAULT_CONFIG = "batched"
WORKLOAD = CONFIGS[DEFAULT_CONFIG]["workload"]
W, H = 800, 800          # mid-size view size

# Per-pair operation model of the render kernels (three sub-samples, depth and normal on),
# counted from the kernel source: an IEEE division is one MUFU reciprocal and 4 FP32 ops,
# expf one MUFU ex2 and 3 FP32 ops, rsqrtf one MUFU op; FFMA, FADD, FMUL and FMNMX one FP32
# op each.  "eval": a (pixel, record) pair that reaches the SDF evaluation (slab test twice,
# entry point and three sub-steps of trilinear SDF and logistic CDF, local and total alpha);
# "acc": the extra work of a pair with alpha >= MIN_ALPHA (compositing, depth, normal; in the
# adjoint the transmittance recovery, normal chain rule, alpha and depth sub-segment
# derivatives over four re-evaluated points, and the colour terms).
OPS_PER_PAIR = {"fwd": {"eval": (269, 16), "acc": (53, 1)},
                "bwd": {"eval": (157, 6), "acc": (527, 24)}}
SMS, FP32_LANES, MUFU_LANES = 148, 128, 16
# DRAM bytes per record (dram__bytes_read.sum + dram__bytes_write.sum of one launch over the
# records it processes: R for the forward, R' for the adjoint), from the ncu capture of the
# batched scene's first 8 views (36.3M records, 29.8M up to the tiles' last contributors):
# forward 4.461 GB (1.17 GB of it the candidate rows it writes for the adjoint), adjoint
# 4.406 GB (0.94 GB of it those rows read back).  A full 64-view launch is too large to
# capture, so its traffic is this figure times its record count (pixels and records grow
# together).
TRAFFIC_PER_RECORD = {"render_fwd_kernel": 4.461e9 / 36327542, "render_bwd_kernel": 4.406e9 / 29848094}


def rank_cameras(rank=0, n_views=None, config=DEFAULT_CONFIG):
    """The views of one rank (data parallel over views, weak scaling): rank r takes the r-th
    block of the workload's views-per-GPU from a camera set of (r + 1) blocks."""
    from svraster_b200 import synthetic as S
    n = CONFIGS[config]["views"]
    if config == "batched":
        cams = S.mixed_resolution_cameras(n * (rank + 1), 3.0, seed=0)[n * rank:n * (rank + 1)]
    elif config == "full":
        cams = S.room_cameras(n * (rank + 1), 1024, 768, seed=0)[n * rank:n * (rank + 1)]
    else:
        cams = S.fibonacci_cameras(n * (rank + 1), 3.0, W, H, fovx_deg=50.0)[n * rank:n * (rank + 1)]
    return cams[:n_views or n]


def make_workload(rank=0, n_views=None, config=DEFAULT_CONFIG):
    from svraster_b200 import synthetic as S
    scene = {"batched": S.scene_batched, "mid": S.scene_mid, "full": S.scene_full}[config](seed=0)
    return scene, rank_cameras(rank, n_views, config)


def max_over_ranks(ms, device):
    """The slowest rank's time: every rank's timed region ends at the same barrier, so the
    job's step time is the maximum (one all-reduce, the same collective on every rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- our arm
def compute_ceiling(state, s_val, kname, kms, sm_mhz):
    """FP32 / MUFU issue ceiling of the dominant render kernel: the pairs it evaluates and
    accepts (counted on the device by the counting instance of the forward), times the
    per-pair operation model OPS_PER_PAIR, over the B200's FP32 lanes (148 SMs x 128) and MUFU
    lanes (148 SMs x 16) at the sampled SM clock."""
    n_eval, n_acc, n_eval_last = state.count_pairs(s_val)
    pas = "bwd" if kname == "render_bwd_kernel" else "fwd"
    ev = n_eval_last if pas == "bwd" else n_eval
    m = OPS_PER_PAIR[pas]
    fp32 = ev * m["eval"][0] + n_acc * m["acc"][0]
    mufu = ev * m["eval"][1] + n_acc * m["acc"][1]
    hz = (sm_mhz or 1965.0) * 1e6
    t_fp32 = fp32 / (SMS * FP32_LANES * hz) * 1e3
    t_mufu = mufu / (SMS * MUFU_LANES * hz) * 1e3
    t_bound = max(t_fp32, t_mufu)
    return {"pairs_evaluated": int(ev), "pairs_accepted": int(n_acc),
            "pairs_evaluated_forward": int(n_eval),
            "fp32_ops": int(fp32), "mufu_ops": int(mufu),
            "fp32_peak_ops_per_s": SMS * FP32_LANES * hz, "mufu_peak_ops_per_s": SMS * MUFU_LANES * hz,
            "sm_mhz": sm_mhz, "t_fp32_ms": round(t_fp32, 4), "t_mufu_ms": round(t_mufu, 4),
            "binding": "fp32" if t_fp32 >= t_mufu else "mufu", "frac": round(t_bound / kms, 4),
            "model": "OPS_PER_PAIR in bench.py (per-pair FP32 and MUFU operations counted from the kernel source)"}


def run_ours(args, rank, world, config):
    from svraster_b200.step import BatchedTrainStep
    import torch
    import torch.distributed as dist
    from svraster_b200 import _lib

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    scene, cams = make_workload(rank, args.views, config)
    workload = CONFIGS[config]["workload"]
    step = BatchedTrainStep(scene, cams, device=dev, lambda_R_concen=0.1)
    L = _lib.load()

    # data parallel over views: the gradients are summed across ranks between the adjoints
    # and Adam (the one exchange step of the path)
    def allreduce_grads(grads):
        dist.all_reduce(step.grad_flat)           # grid, sh0 and shs gradients in one call
    hook = allreduce_grads if world > 1 else None
    use_graph = not args.no_graph
    for _ in range(args.warmup):
        step.step(grad_hook=hook)
    # the render launch configuration is chosen on this batch before anything is timed
    tuned = None
    if not args.no_autotune:
        tuned = step.autotune()
        step.step(grad_hook=hook)   # the tuner reused the gradient buffers: one clean step
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    def timed(fn, n):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = L.svr_kernel_launches()
        with ClockSampler(dev.index) as clk:
            torch.cuda.synchronize()
            ev0.record()
            for _ in range(n):
                fn()
            ev1.record()
            torch.cuda.synchronize()
        return ev0.elapsed_time(ev1), L.svr_kernel_launches() - n0, clk.summary()

    # eager steps, every stage bracketed by events (the per-stage breakdown)
    step_events = []

    def eager():
        step.step(time_render=True, grad_hook=hook)
        step_events.append(step.ev)
    n_eager = max(3, min(args.steps, 10))
    eager_ms, launches, clocks = timed(eager, n_eager)
    stages = [BatchedTrainStep.stage_ms(m) for m in step_events]
    stage_avg = {k: float(np.mean([s_[k] for s_ in stages])) for k in stages[0]}
    fwd_ms = [s_["render_fwd"] for s_ in stages]
    bwd_ms = [s_["render_bwd"] for s_ in stages]
    total_ms = eager_ms * args.steps / n_eager
    graph_info = None
    if use_graph:
        # the whole step, all-reduce included when several ranks run, as one CUDA graph
        per_step = step.capture(grad_hook=hook)
        for _ in range(args.warmup):
            step.replay()
        total_ms, _, clocks = timed(step.replay, args.steps)
        launches = per_step * args.steps
        st_raster, st_misc = step.graph_status()
        if st_raster or st_misc:
            raise RuntimeError(f"graph replay status raster={st_raster} misc={st_misc}")
        graph_info = {"captured": True, "kernels_per_step": per_step, "record_capacity": step.capacity,
                      "allreduce_in_graph": world > 1, "eager_ms_per_step": round(eager_ms / n_eager, 3)}
    else:
        launches = launches * args.steps // n_eager

    if world > 1:
        total_ms = max_over_ranks(total_ms, dev)
        dist.barrier()
    ms_per_step = total_ms / args.steps
    rays = step.rays * world
    value = rays / (ms_per_step * 1e-3) / 1e6

    # roofline of the dominant kernel (algorithmic bytes of the reference's per-record layout)
    R, R_prime = step.record_counts()
    nd = step.state.geom_fields()[0]
    V_vis = int((nd.view(len(cams), -1) > 0).any(0).sum().item())
    P = step.P
    fwd_avg, bwd_avg = float(np.mean(fwd_ms)), float(np.mean(bwd_ms))
    fwd_bytes = R * 72 + P * 52
    bwd_bytes = R_prime * 72 + P * 68 + V_vis * 48
    if bwd_avg >= fwd_avg:
        kname, kbytes, kms = "render_bwd_kernel", bwd_bytes, bwd_avg
    else:
        kname, kbytes, kms = "render_fwd_kernel", fwd_bytes, fwd_avg
    peak, peak_src = measured_peaks()
    achieved = kbytes / (kms * 1e-3) / 1e9
    compute = compute_ceiling(step.state, step.s_val, kname, kms, clocks.get("sm_mhz"))
    roofline = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1), "peak": peak,
                "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": int(TRAFFIC_PER_RECORD[kname] * (R_prime if kname == "render_bwd_kernel" else R)),
                "traffic_note": "DRAM bytes per record of an ncu capture of 8 views of the batched scene, "
                                "times this launch's records (TRAFFIC_PER_RECORD)",
                "algorithmic_bytes": int(kbytes), "launch_ms": round(kms, 4),
                "launch_ms_source": "CUDA events around the kernel in eager steps, on its stream",
                "compute": compute}

    result = {"metric": "fwd+bwd Mrays/s", "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
              "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
              "iters_per_s": round(1e3 / ms_per_step, 3),
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
              "data": "synthetic (seeded procedural scene, N(0,1) upstream gradients)",
              "config": {"workload": workload, "n_voxels": scene.n_vox, "n_grid_pts": int(step.grid.numel()),
                         "views_per_gpu": len(cams), "image": CONFIGS[config]["image"], "rays_per_step": rays,
                         "records_R": R, "records_R_prime": R_prime, "visible_voxels": V_vis,
                         "l2": "inputs larger than L2 (records + SH state > 126 MB)",
                         "parallelism": f"dp{world} over views" if world > 1 else "single GPU"},
              "stages_ms": {k: round(v, 3) for k, v in stage_avg.items()},
              "roofline": roofline, "gpu_launches": int(launches), "clocks": clocks,
              "cuda_graph": graph_info or {"captured": False},
              "autotuned_render": ({k: tuned[k] for k in ("fwd_config", "bwd_config", "ms")} if tuned
                                   else "default configuration")}
    return result, step, scene, cams


def run_e2e_batched(args, scene, cams, dev):
    """The same metric through the batched C-ABI path (svraster_b200.step.BatchedTrainStep,
    the step as a forward graph and two backward graphs) with host-resident inputs: every step
    copies a step's upstream gradient planes and target image (dL/dcolor, dL/ddepth,
    dL/dnormal, gt; 13 floats per pixel) from pinned host memory on a copy stream, one step
    ahead into the other of two plane sets, and reads every step's mean transmittance back
    (through a pinned slot, one step later, so the host does not stall the stream)."""
    import torch
    from svraster_b200.step import BatchedTrainStep
    step = BatchedTrainStep(scene, cams, device=dev, lambda_R_concen=0.1)
    rng = np.random.default_rng(1)
    P = step.P
    host = [torch.from_numpy(rng.normal(size=n * P).astype(np.float32)).pin_memory() for n in (3, 4, 3)]
    host.append(torch.from_numpy(rng.uniform(size=3 * P).astype(np.float32)).pin_memory())
    h2d = sum(h.numel() * 4 for h in host)
    for _ in range(args.warmup):
        step.step()
    # two sets of upstream planes, one backward graph each: the copies of step k+1's planes
    # into one set overlap the whole of step k, whose adjoint reads the other set
    step.capture(split=True, upstream_sets=2)
    copy_stream = torch.cuda.Stream(device=dev)
    done = [torch.cuda.Event(), torch.cuda.Event()]     # set i free again (its adjoint ran)
    filled = [torch.cuda.Event(), torch.cuda.Event()]   # set i holds its step's planes
    k = [0]

    def fill(i):
        copy_stream.wait_event(done[i])
        with torch.cuda.stream(copy_stream):
            for hsrc, ddst in zip(host, step.upstream(i)):
                ddst.copy_(hsrc, non_blocking=True)
        filled[i].record(copy_stream)

    # each step's result (mean transmittance) goes to a pinned host slot and is read one step
    # later, once its event has completed, so the host never stalls the stream on it
    res_host = torch.zeros(2, dtype=torch.float32).pin_memory()
    res_ready = [torch.cuda.Event(), torch.cuda.Event()]
    results = []

    def one_step():
        i = k[0] % 2
        compute = torch.cuda.current_stream(dev)
        fill(1 - i)                               # the next step's planes, during this step
        step.replay_forward()
        compute.wait_event(filled[i])
        _, T = step.replay_backward(i)
        done[i].record(compute)
        res_host[i:i + 1].copy_(T.mean().reshape(1), non_blocking=True)
        res_ready[i].record(compute)
        if k[0] > 0:                              # device -> host read of the previous step's result
            res_ready[1 - i].synchronize()
            results.append(float(res_host[1 - i]))
        k[0] += 1

    def drain():
        last = (k[0] - 1) % 2
        res_ready[last].synchronize()
        results.append(float(res_host[last]))

    for e in done:
        e.record(torch.cuda.current_stream(dev))
    fill(0)
    for _ in range(3):
        one_step()
    drain()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        one_step()
    drain()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    assert len(results) == 4 + args.steps and all(np.isfinite(results))
    status = step.graph_status()
    del step
    torch.cuda.empty_cache()
    return {"value": round(P / (ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "ms_per_step": round(ms, 3),
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 4, "graph_status": list(status),
            "path": "svraster_b200.step.BatchedTrainStep (C ABI, forward / backward graphs), "
                    "upstream planes from pinned host memory every step, mean T read back"}


def run_native_step(args, scene, cams, dev):
    """The batched step issued by the library's own host code (svr_step_create / svr_step_capture
    / svr_step_run through ``native_step.NativeStep``; what a host without Python runs): the
    same launches as the headline's step, recorded by the library into two CUDA graphs and
    launched on the caller's stream, inputs resident in HBM, same timing as ``value``."""
    import torch
    from svraster_b200.native_step import NativeStep
    ns = NativeStep(scene, cams, device=dev)
    g = torch.Generator(device=dev).manual_seed(0)
    for name in ("dcolor", "ddepth", "dnormal"):
        buf = ns.buffer(name)
        buf.copy_(torch.randn(buf.numel(), device=dev, generator=g))
    kernels = ns.capture()
    for _ in range(args.warmup):
        ns.run()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        ns.run()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    info, status = ns.info(), ns.status()
    ns.close()
    del ns
    torch.cuda.empty_cache()
    return {"value": round(info["pixels"] / (ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "ms_per_step": round(ms, 3),
            "kernels_per_step": int(kernels), "records": info["capacity"], "status": list(status),
            "path": "svr_step_create / svr_step_capture / svr_step_run (C ABI, the library's own graphs)"}


def run_per_view(args, scene, cams, dev, host_inputs, steps=None, warmup=None):
    """The same step through the plain per-view path: the drop-in API (renderer.rasterize_voxels
    with autograd, GatherGeoParams, SH_eval) one view at a time, as the reference's train.py
    drives its extension, then grid_loss_bw and SparseAdam.  ``host_inputs``: every step copies
    all views' upstream planes and target images from pinned host memory (view v's render waits
    only for its own planes) and reads the step's result back; otherwise the planes stay
    resident on the device, as for the batched ``value``."""
    import torch
    from svraster_b200 import renderer, grid_loss_bw
    from svraster_b200.sparse_adam import SparseAdam

    steps = steps or args.steps
    warmup = warmup or args.warmup
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    octpath = t(scene.octpath, torch.int64)
    centers = t(scene.vox_center)
    lengths = t(scene.vox_size)
    is_leaf = t(scene.is_leaf, torch.uint8)
    vox_key = t(scene.vox_key, torch.int64)
    grid = t(scene.geo_grid_pts).requires_grad_(True)
    sh0 = t(scene.sh0).requires_grad_(True)
    shs = t(scene.shs).requires_grad_(True)
    log_s = torch.tensor([scene.log_s], dtype=torch.float32, device=dev).requires_grad_(True)
    vox_size_inv = 1.0 / lengths
    opt = SparseAdam([{"params": [grid], "lr": 1e-3}, {"params": [sh0], "lr": 1e-3}, {"params": [shs], "lr": 1e-4}],
                     betas=(0.1, 0.99), eps=1e-15)

    def vox_fn(idx, cam_pos, color_mode):
        geos = renderer.GatherGeoParams.apply("triinterp3", vox_key, vox_size_inv, idx, grid)
        rgbs = renderer.SH_eval.apply(3, idx, centers, cam_pos, None, sh0, shs)
        return {"geos": geos, "rgbs": rgbs, "subdiv_p": torch.zeros(scene.n_vox, 1, device=dev), "log_s": log_s}

    rng = np.random.default_rng(0)
    host = []
    for c in cams:
        P = c.width * c.height
        planes = [torch.from_numpy(rng.normal(size=n * P).astype(np.float32)) for n in (3, 4, 3)]
        gt = torch.from_numpy(rng.uniform(size=3 * P).astype(np.float32))
        if host_inputs:
            planes, gt = [p_.pin_memory() for p_ in planes], gt.pin_memory()
        host.append((planes, gt))
    mats = [(t(c.w2c), t(c.c2w)) for c in cams]
    bg = torch.zeros(3, device=dev)
    # dense-grid table (static between prune / subdivide)
    from svraster_b200 import utils
    res_pow2 = min(int(scene.octlevel.max()), 9)
    res = 1 << res_pow2
    mask, keys, g2v = utils.valid_gradient_table(centers, lengths, torch.zeros(3, device=dev), scene.scene_extent,
                                                 res_pow2, is_leaf)
    ext = np.float32(scene.scene_extent)
    coord = t(np.round(((scene.vox_center - scene.vox_size * np.float32(0.5)) + ext * np.float32(0.5)) / ext
                       * np.float32(res)))
    vsize = t(np.round(scene.vox_size / ext * np.float32(res))).reshape(-1)
    active = torch.arange(keys.numel(), dtype=torch.int32, device=dev)
    h2d = sum(sum(p_.numel() for p_ in planes) * 4 + gt.numel() * 4 for planes, gt in host) + 2 * 64 * len(cams)

    # device buffers of the upstream planes; with host inputs they are refilled every step on a
    # copy stream, otherwise filled once
    dev_bufs = [([p_.to(dev) for p_ in planes], gt.to(dev)) for planes, gt in host]
    copy_stream = torch.cuda.Stream(device=dev)

    def one_step(it):
        opt.zero_grad(set_to_none=False) if grid.grad is not None else None
        tot = torch.zeros((), device=dev)
        compute = torch.cuda.current_stream(dev)
        ready = [None] * len(cams)
        if host_inputs:
            copy_stream.wait_stream(compute)      # buffers are free once the last step used them
            with torch.cuda.stream(copy_stream):
                for v, ((planes, gt_h), (dplanes, dgt)) in enumerate(zip(host, dev_bufs)):
                    for hp, dp in zip(planes, dplanes):
                        dp.copy_(hp, non_blocking=True)
                    dgt.copy_(gt_h, non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(copy_stream)
                    ready[v] = ev
        for (dplanes, dgt), ev, (w2c, c2w), c in zip(dev_bufs, ready, mats, cams):
            if ev is not None:
                compute.wait_event(ev)
            dc, dd, dn = dplanes
            gt = dgt.view(3, c.height, c.width)
            rs = renderer.RasterSettings(color_mode="sh", vox_geo_mode="triinterp3", density_mode="sdf",
                                         image_width=c.width, image_height=c.height, tanfovx=c.tanfovx,
                                         tanfovy=c.tanfovy, cx=c.cx, cy=c.cy, w2c_matrix=w2c, c2w_matrix=c2w,
                                         background=bg, near=c.near, need_depth=True, need_normal=True,
                                         lambda_R_concen=0.1, gt_color=gt)
            color, depth, normal, T, _, _ = renderer.rasterize_voxels(rs, octpath, centers, lengths, vox_fn, is_leaf)
            torch.autograd.backward([color, depth, normal],
                                    [dc.view(3, c.height, c.width), dd.view(4, c.height, c.width),
                                     dn.view(3, c.height, c.width)])
            tot = tot + T.detach().mean()
        for fn in (grid_loss_bw.laplacian_smoothness, grid_loss_bw.grid_eikonal):
            fn(grid, vox_key, coord, vsize, res, mask, keys, g2v, active, 1e-3, float(res) / scene.scene_extent,
               True, False, grid.grad, seed=it)
        opt.step()
        return float(tot.item()) if host_inputs else tot   # device -> host read of the step's result

    for i in range(warmup):
        one_step(i)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for i in range(steps):
        one_step(1000 + i)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    rays = sum(c.width * c.height for c in cams)
    out = {"value": round(rays / (ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "ms_per_step": round(ms, 3),
           "iters_per_s": round(1e3 / ms, 3), "steps": steps,
           "path": "svraster_b200.renderer.rasterize_voxels per view + autograd + grid_loss_bw + SparseAdam"}
    if host_inputs:
        out.update({"h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 4})
    del opt, grid, sh0, shs, dev_bufs
    torch.cuda.empty_cache()
    return out


class StdoutToStderr:
    """Sends everything written to file descriptor 1 (C printf included) to descriptor 2 while
    active, so that the bench's JSON line stays the only thing on stdout."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def reference_extension():
    """The reference's own CUDA extension (oracle/_ref/svraster_ref_C.so, built from its
    unmodified sources by oracle/build_ref.py), or None where it was not built."""
    import importlib.util
    so = os.path.join(ROOT, "oracle", "_ref", "svraster_ref_C.so")
    if not os.path.exists(so):
        return None
    spec = importlib.util.spec_from_file_location("svraster_ref_C", so)
    mod = importlib.util.module_from_spec(spec)
    with StdoutToStderr():
        spec.loader.exec_module(mod)
    return mod


REF_UNAVAILABLE = {"unavailable": "the reference extension was not built (oracle/build_ref.py needs the reference "
                                  "sources on the build machine)"}


def run_reference_cuda(scene, cams, dev, steps=3, warmup=1):
    """See _run_reference_cuda; the reference extension prints to stdout (valid_gradient_table),
    which is kept off the bench's stdout."""
    with StdoutToStderr():
        return _run_reference_cuda(scene, cams, dev, steps, warmup)


def _run_reference_cuda(scene, cams, dev, steps=3, warmup=1):
    """The reference's own CUDA extension (oracle/_ref, built from its unmodified sources by
    oracle/build_ref.py) on the same scene and views, one view at a time on the default stream
    as the reference's train.py drives it (train.py:316-709): per view rasterize_preprocess,
    gather and SH on the in-frustum voxels, rasterize_voxels, rasterize_voxels_backward and
    the gather / SH adjoints; per step the Laplacian and grid-Eikonal adjoints over every
    dense-grid key and Adam on grid / sh0 / shs.  A baseline leg, timed after our own timed
    regions with CUDA events (median step).  Returns {"unavailable": why} when the built
    extension is not present."""
    import torch
    R_ = reference_extension()
    if R_ is None:
        return dict(REF_UNAVAILABLE)
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
    octpath, centers, lengths = t(scene.octpath, torch.int64), t(scene.vox_center), t(scene.vox_size)
    is_leaf = t(scene.is_leaf, torch.uint8)
    vox_key, grid = t(scene.vox_key, torch.int64), t(scene.geo_grid_pts)
    sh0, shs = t(scene.sh0), t(scene.shs)
    s_val = torch.exp(torch.tensor([scene.log_s], dtype=torch.float32, device=dev) * 10.0)
    views = [(t(c.w2c), t(c.c2w), c) for c in cams]
    bg = torch.zeros(3, device=dev)
    g = torch.Generator(device=dev).manual_seed(0)
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
    params = [grid, sh0, shs]
    ms_ = [torch.zeros_like(p_) for p_ in params]
    vs_ = [torch.zeros_like(p_) for p_ in params]

    def one_step(it):
        dgrid = torch.zeros_like(grid)
        dsh0 = torch.zeros_like(sh0)
        dshs = torch.zeros_like(shs)
        for (w2c, c2w, c), (dc, dd, dn, dT, gt) in zip(views, ups):
            ndup, geom = R_.rasterize_preprocess(c.width, c.height, c.tanfovx, c.tanfovy, c.cx, c.cy, w2c, c2w, 0,
                                                 c.near, octpath, centers, lengths, is_leaf, False)
            care = torch.where(ndup > 0)[0]
            geos = R_.gather_triinterp_geo_params(vox_key, care, grid)
            cam_pos = c2w[:3, 3].contiguous()
            rgbs = R_.sh_compute(3, care, centers, cam_pos, sh0, shs)
            out = R_.rasterize_voxels(3, 1, c.width, c.height, c.tanfovx, c.tanfovy, c.cx, c.cy, w2c, c2w, bg, 0,
                                      True, False, True, False, octpath, centers, lengths, geos, rgbs,
                                      torch.empty(scene.n_vox, 0, device=dev), geom, False, s_val)
            nr, binning, img, color, depth, normal, T = out[:7]
            dgeos, drgbs, _, ds = R_.rasterize_voxels_backward(
                nr, 3, 1, c.width, c.height, c.tanfovx, c.tanfovy, c.cx, c.cy, w2c, c2w, bg, octpath, centers,
                lengths, geos, rgbs, geom, binning, img, T, dc, dd, dn, dT, 0.1, gt, 0.0, 0.0, True, True, depth,
                normal, False, s_val, out[8])
            dgrid += R_.gather_triinterp_geo_params_bw(vox_key, care, grid.numel(), dgeos.contiguous())
            a0, a1 = R_.sh_compute_bw(3, 16, care, centers, cam_pos, rgbs, drgbs.contiguous())
            dsh0 += a0
            dshs += a1
        R_.laplacian_smoothness_bw(grid, vox_key, coord, vsize, res, mask, keys, g2v, active, 1e-3,
                                   float(res) / scene.scene_extent, True, False, dgrid)
        R_.grid_eikonal_bw(grid, vox_key, coord, vsize, res, mask, keys, g2v, active, 1e-3,
                           float(res) / scene.scene_extent, True, False, dgrid)
        for p_, gr, m, v, lr in zip(params, (dgrid, dsh0, dshs), ms_, vs_, (1e-3, 1e-3, 1e-4)):
            R_.unbiased_adam_step(False, p_, gr, m, v, it + 1, lr, 0.1, 0.99, 1e-15)

    for i in range(warmup):
        one_step(i)
    torch.cuda.synchronize()
    times = []
    for i in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        one_step(warmup + i)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    rays = sum(c.width * c.height for c in cams)
    del params, ms_, vs_, ups
    torch.cuda.empty_cache()
    return {"value": round(rays / ms / 1e3, 3), "unit": "Mrays/s", "ms_per_step": round(ms, 3),
            "iters_per_s": round(1e3 / ms, 4), "steps": steps,
            "path": "reference svraster_cuda._C built from its unmodified sources, per view, default stream"}


def run_extraction(step, scene, cams, dev):
    """TSDF fusion of the 8 rendered median-depth maps into every grid point (one launch) and
    marching cubes over every voxel of the trained SDF (extract_mesh_sdf.py:337-381 path),
    timed with CUDA events; CPU baseline: the NumPy restatement on a sample."""
    import torch
    from svraster_b200 import _lib
    from svraster_b200._lib import check, ptr, stream_ptr
    from svraster_b200.marching_cubes import torch_marching_cubes_grid
    from svraster_b200.raster import RasterState
    st_ = RasterState(step.views, step.N, dev)
    st_.preprocess(step.octpath, step.centers, step.lengths, step.is_leaf)
    st_.bin(step.octpath)
    color, depth, normal, T, _ = st_.render(3, True, False, step.centers, step.lengths, step.geos, step.rgbs,
                                            step.s_val, rgb_per_view=True)
    xyz = torch.as_tensor(scene.grid_pts_xyz).to(dev).contiguous()
    M = xyz.shape[0]
    finest = scene.scene_extent * 2.0 ** -int(scene.octlevel.max())
    trunc = 3.0 * finest
    wacc = torch.zeros(M, device=dev)
    sacc = torch.zeros(M, device=dev)
    proj = []
    for c in cams:
        proj += [c.tanfovx, c.tanfovy, 0.5, 0.5]
    proj_h = (len(proj) * _lib.C.c_double)(*proj)
    L = _lib.load()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for rep in range(2):   # first pass warms up
        wacc.zero_(); sacc.zero_()
        torch.cuda.synchronize()
        e[0].record()
        check(L.svr_tsdf_integrate(st_.views, proj_h, len(cams), M, ptr(xyz), ptr(depth), 4, 2, ptr(T), 1, 0, 1, None,
                                   trunc, 0.01, 0.5, 1, 0, 0, 10.0, 0, ptr(wacc), ptr(sacc), stream_ptr(dev)), "tsdf")
        e[1].record()
        grid_val = step.grid.reshape(-1)
        v, f = torch_marching_cubes_grid(grid_val, xyz, step.vox_key, 0.0)
        e[2].record()
        torch.cuda.synchronize()
    tsdf_ms, mc_ms = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    fused = int((wacc > 0).sum().item())
    # CPU baseline: NumPy restatements on a sample (one view of TSDF, 1/16 of the voxels for MC)
    from oracle import extract_oracle as X
    d0 = depth[: 4 * cams[0].width * cams[0].height].view(4, cams[0].height, cams[0].width)[2].cpu().numpy()
    a0 = (1 - T[: cams[0].width * cams[0].height]).view(cams[0].height, cams[0].width).cpu().numpy()
    wc = np.zeros((M, 1), np.float32); sc_ = np.zeros((M, 1), np.float32)
    t0 = time.perf_counter()
    X.tsdf_integrate(wc, sc_, scene.grid_pts_xyz, cams[0].w2c, cams[0].c2w, cams[0].tanfovx, cams[0].tanfovy, 0.5,
                     0.5, d0, a0, trunc, crop_border=0.01)
    cpu_tsdf = time.perf_counter() - t0
    sub = scene.vox_key[::16]
    t0 = time.perf_counter()
    X.marching_cubes(step.grid.reshape(-1).cpu().numpy(), scene.grid_pts_xyz, sub, 0.0)
    cpu_mc = time.perf_counter() - t0
    return {"tsdf_ms": round(tsdf_ms, 3), "tsdf_views": len(cams), "grid_points": M, "fused_points": fused,
            "tsdf_Mpoint_views_per_s": round(M * len(cams) / tsdf_ms / 1e3, 1),
            "mc_ms": round(mc_ms, 3), "mc_voxels": scene.n_vox, "mc_faces": int(f.shape[0]),
            "mc_Mvoxels_per_s": round(scene.n_vox / mc_ms / 1e3, 1),
            "cpu_numpy_restatement": {"tsdf_Mpoint_views_per_s": round(M / cpu_tsdf / 1e6, 3),
                                      "mc_Mvoxels_per_s": round(len(sub) / cpu_mc / 1e6, 3), "cores": 1,
                                      "sample": f"TSDF: 1 of {len(cams)} views; MC: every 16th voxel"}}


def run_adaptive(step, scene, cams, dev):
    """Subdivision support and training statistics on the bench scene: the grid-point link over
    all voxels, subdivision of 5% of the voxels (children, trilinear corner values, relink,
    mean aggregation), and the training statistics over the batch's views, each timed with
    CUDA events beside the PyTorch calls the reference makes for the same results
    (unique(dim=0, return_inverse=True), index_reduce_ mean; src/utils/octree_utils.py:203-222,
    src/sparse_voxel_gears/adaptive.py:349-411)."""
    import torch
    from svraster_b200 import adaptive as A
    octpath = step.octpath.reshape(-1, 1)
    octlevel = torch.as_tensor(scene.octlevel.reshape(-1, 1).astype(np.int8), device=dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=3):
        fn()
        ts = []
        for _ in range(reps):
            a, b = ev(), ev()
            a.record(); fn(); b.record(); torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    shift = torch.tensor([[(k >> 2) & 1, (k >> 1) & 1, k & 1] for k in range(8)], dtype=torch.int64, device=dev)

    def torch_link():
        from svraster_b200 import utils
        ijk = utils.octpath_2_ijk(octpath, octlevel)
        lv2 = (16 - octlevel).long()
        g = ((ijk << lv2).view(-1, 1, 3) + (shift << lv2.view(-1, 1, 1))).reshape(-1, 3)
        return g.unique(dim=0, return_inverse=True)

    link_ms = timed(lambda: A.build_grid_pts_link(octpath, octlevel))
    link_torch_ms = timed(torch_link, reps=1)
    key, vkey = A.build_grid_pts_link(octpath, octlevel)
    vals = step.grid.reshape(-1)[vkey].unsqueeze(-1).contiguous()
    M = len(key)

    def torch_agg():
        import warnings
        out = torch.zeros(M, 1, device=dev)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")   # index_reduce_ is marked beta
            out.index_reduce_(0, vkey.reshape(-1), vals.reshape(-1, 1), "mean", include_self=False)
        return out
    agg_ms = timed(lambda: A.agg_voxel_into_grid_pts(M, vkey, vals))
    agg_torch_ms = timed(torch_agg)
    sel = torch.arange(0, scene.n_vox, 20, device=dev)
    interp_ms = timed(lambda: A.subdivide_by_interp(vals[sel]))
    geos = step.grid.reshape(-1)[step.vox_key]
    stat_ms = timed(lambda: A.compute_training_stat(cams, octpath, step.centers, step.lengths, step.is_leaf, geos,
                                                    step.s_val), reps=2)
    return {"voxels": scene.n_vox, "grid_points": M,
            "grid_link_ms": round(link_ms, 3), "grid_link_torch_unique_ms": round(link_torch_ms, 3),
            "agg_mean_ms": round(agg_ms, 3), "agg_mean_torch_index_reduce_ms": round(agg_torch_ms, 3),
            "subdivide_interp_ms_5pct": round(interp_ms, 3),
            "training_stat_ms": round(stat_ms, 3), "training_stat_views": len(cams)}


REG_POINTS = 1 << 21


def regulariser_inputs(scene, grid_mask, res, dev):
    """Seeded inputs of the regulariser timings: a random half of the voxels active for the
    voxel Eikonal (randperm(N)[:N/2], the default drop ratio 0.5 of train.py:562-564), 1/size
    per voxel, and 2M points (grid units) uniform inside the masked cells for the points loss."""
    import torch
    g = torch.Generator(device=dev).manual_seed(5)
    cells = torch.nonzero(grid_mask.reshape(-1)).reshape(-1)
    pick = cells[torch.randint(0, cells.numel(), (REG_POINTS,), device=dev, generator=g)]
    ijk = torch.stack([pick % res, (pick // res) % res, pick // (res * res)], 1).float()
    pts = (ijk + torch.rand(REG_POINTS, 3, device=dev, generator=g)).contiguous()
    vsi = (1.0 / torch.as_tensor(scene.vox_size.reshape(-1), device=dev)).contiguous()
    active = torch.randperm(scene.n_vox, device=dev, generator=g)[:scene.n_vox // 2].to(torch.int32).contiguous()
    return active, vsi, pts


def run_regularisers(step, scene, dev):
    """Voxel Eikonal, sign total variation (dense and tv_sparse) and the points loss on the
    bench scene through the drop-in grid_loss_bw calls: CUDA events around 10 back-to-back
    calls (the per-call host work overlaps the GPU), median of 5.  The voxel Eikonal and total
    variation run with the voxels visited in spatial order (the default; the one-off order
    build per octree is timed apart) and in storage order as the reference visits them.  Compulsory HBM bytes: per
    voxel (active voxel for the voxel Eikonal) its 8 corner keys (64 B), 1/size (4 B) and its
    active index (4 B, voxel Eikonal); per grid point one SDF read (4 B) and one gradient
    read-modify-write (8 B)."""
    import torch
    from svraster_b200 import grid_loss_bw as GL
    peak, _ = measured_peaks()
    res = 1 << step.res_pow2
    active, vsi, pts = regulariser_inputs(scene, step.grid_mask, res, dev)
    N, M = scene.n_vox, step.grid.shape[0]
    grad = torch.zeros_like(step.grid)

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
        return float(np.median(ts))

    def order_build():
        GL._ORDER_CACHE.clear()
        GL.voxel_order(step.vox_key, M)
    order_ms = timed(order_build, calls=1)
    out = {"voxels": N, "active_voxels": active.numel(), "grid_points": M, "points": REG_POINTS,
           "voxel_order_build_ms": round(order_ms, 4)}
    vg_bytes, tv_bytes = active.numel() * 72 + M * 12, N * 68 + M * 12
    for form, ordered in (("", True), ("_storage_order", False)):
        vg_ms = timed(lambda: GL.voxel_gradient(step.grid, step.vox_key, vsi, active, 1e-3, False, False, grad,
                                                ordered=ordered))
        tv_ms = timed(lambda: GL.total_variation(step.grid, step.vox_key, 1e-3, vsi, False, False, grad,
                                                 ordered=ordered))
        tvs_ms = timed(lambda: GL.total_variation(step.grid, step.vox_key, 1e-3, vsi, False, True, grad,
                                                  ordered=ordered))
        out.update({f"voxel_gradient{form}_ms": round(vg_ms, 4),
                    f"voxel_gradient{form}_frac": round(vg_bytes / vg_ms / 1e6 / peak, 3),
                    f"total_variation{form}_ms": round(tv_ms, 4),
                    f"total_variation{form}_frac": round(tv_bytes / tv_ms / 1e6 / peak, 3),
                    f"total_variation_sparse{form}_ms": round(tvs_ms, 4)})
    pl_ms = timed(lambda: GL.points_loss(pts, step.grid, step.vox_key, step.grid_voxel_coord, step.grid_voxel_size,
                                         res, step.grid_mask, step.grid_keys, step.grid2voxel, 1e-3, 1.0, True,
                                         False, grad))
    out.update({"points_loss_ms": round(pl_ms, 4), "points_loss_Mpoints_per_s": round(REG_POINTS / pl_ms / 1e3, 1),
                "compulsory_bytes": {"voxel_gradient": vg_bytes, "total_variation": tv_bytes}})
    # the reference's own extension on the same inputs, timed the same way
    R_ = reference_extension()
    if R_ is None:
        out["reference_cuda"] = dict(REF_UNAVAILABLE)
    else:
        with StdoutToStderr():
            ref = {"voxel_gradient_ms": timed(lambda: R_.voxel_gradient_bw(step.grid, step.vox_key, vsi, active, 1e-3,
                                                                           False, False, grad)),
                   "total_variation_ms": timed(lambda: R_.total_variation_bw(step.grid, step.vox_key, 1e-3, vsi,
                                                                             False, False, grad)),
                   "total_variation_sparse_ms": timed(lambda: R_.total_variation_bw(step.grid, step.vox_key, 1e-3, vsi,
                                                                                    False, True, grad)),
                   "points_loss_ms": timed(lambda: R_.points_loss_bw(pts, step.grid, step.vox_key,
                                                                     step.grid_voxel_coord, step.grid_voxel_size, res,
                                                                     step.grid_mask, step.grid_keys, step.grid2voxel,
                                                                     1e-3, 1.0, True, False, grad))}
        out["reference_cuda"] = {k: round(v, 4) for k, v in ref.items()}
        out["speedup_vs_reference_cuda"] = {k[:-3]: round(v / out[k], 2) for k, v in ref.items() if out.get(k)}
    return out


def run_normal_losses(step, cams, dev):
    """The two normal-from-depth consistency losses with their gradients on the bench batch's
    rendered depth / normal / transmittance planes (one render forward of the step's state;
    all 8 views per launch), CUDA events around 10 back-to-back calls, median of 5.
    Compulsory HBM bytes per pixel: the depth plane (4 B), normal (12 B), T (4 B, mean-depth
    loss only), the depth-gradient plane and the normal gradient read and written (8 + 24 B)."""
    import torch
    from svraster_b200 import loss_utils as LU
    from svraster_b200.raster import RasterState
    peak, _ = measured_peaks()
    state = RasterState(step.views, step.N, dev)
    state.preprocess(step.octpath, step.centers, step.lengths, step.is_leaf)
    state.bin(step.octpath)
    # step.geos / step.rgbs hold the last step's gathered corner values and colours
    _, depth, normal, T, _ = state.render(3, True, True, step.centers, step.lengths, step.geos, step.rgbs,
                                          step.s_val, rgb_per_view=True)
    gd, gn = torch.zeros_like(depth), torch.zeros_like(normal)
    loss = torch.zeros(len(cams), dtype=torch.float64, device=dev)
    P = T.numel()
    out = {"views": len(cams), "pixels": P}
    for name, mode, ks, tol, nbytes in (("mean_depth_ks3_tol90", "dmean", 3, float(np.float32(np.cos(np.pi / 2))), 52),
                                        ("median_depth_ks3", "dmed", 3, -1.0, 48)):
        fn = lambda: LU.normal_depth_loss_views(step.views, depth, normal, T, mode, ks, tol, 1e-3, gd, gn, loss)
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(10):
                fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) / 10)
        ms = float(np.median(ts))
        out[f"{name}_ms"] = round(ms, 4)
        out[f"{name}_frac"] = round(P * nbytes / ms / 1e6 / peak, 3)
    return out


def run_step_with_normal_losses(scene, cams, dev, steps=10):
    """The bench step with both normal-from-depth consistency losses switched on
    (lambda_normal_dmean = lambda_normal_dmed = 0.001, the values train.py:1360-1362 sets),
    graph replays, CUDA events around ``steps`` replays."""
    import torch
    from svraster_b200.step import BatchedTrainStep
    step = BatchedTrainStep(scene, cams, device=dev, lambda_R_concen=0.1,
                            normal_losses=dict(lambda_dmean=1e-3, dmean_ks=3, dmean_tol_deg=90.0, lambda_dmed=1e-3))
    for _ in range(3):
        step.step()
    step.capture()
    for _ in range(3):
        step.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        step.replay()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    out = {"ms_per_step": round(ms, 3), "Mrays_per_s": round(step.P / ms / 1e3, 2),
           "nd_loss_last_step": round(float(step.nd_loss.sum()), 6), "graph_status": list(step.graph_status())}
    del step
    torch.cuda.empty_cache()
    return out


def checkpoint_tensors(scene, dev):
    """The fields of the bench model that a quantized checkpoint codes (io.py:111-114): the SDF
    grid [M,1], sh0 [N,3] and shs [N,15,3], on the device."""
    import torch
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    return {"_geo_grid_pts": t(scene.geo_grid_pts.reshape(-1, 1)), "_sh0": t(scene.sh0), "_shs": t(scene.shs)}


def run_checkpoint(scene, dev):
    """8-bit checkpoint coding of the bench model through svraster_b200.io: quantize_state_dict
    (19 codebooks: the grid, 3 sh0 columns, 15 shs columns; each syncs once per round) and
    dequantize_state_dict, wall clock around a synchronised call, median of 3."""
    import torch
    from svraster_b200 import io
    fields = checkpoint_tensors(scene, dev)

    def timed(fn, reps=3):
        fn()
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3)
        return float(np.median(ts))

    def quant():
        sd = dict(fields)
        io.quantize_state_dict(sd)
        return sd
    q_ms = timed(quant)
    sd = quant()
    d_ms = timed(lambda: io.dequantize_state_dict(dict(sd)))
    n = sum(v.numel() for v in fields.values())
    deq = dict(sd)
    io.dequantize_state_dict(deq)
    err = float(max((deq[k] - fields[k]).abs().mean().item() / fields[k].abs().mean().item() for k in fields))
    out = {"values": n, "codebooks": 1 + fields["_sh0"].shape[1] + fields["_shs"].shape[1],
           "quantize_ms": round(q_ms, 2), "quantize_Mvalues_per_s": round(n / q_ms / 1e3, 1),
           "dequantize_ms": round(d_ms, 3), "mean_rel_abs_error": round(err, 5)}
    # CPU baseline: the reference builds the codebook with torch ops (io.py:123-167), restated
    # bit for bit by the C oracle, timed single-threaded on a sample of the same columns
    from oracle import oracle as O
    cols = [scene.geo_grid_pts.reshape(-1)] + [scene.sh0[:, j] for j in range(scene.sh0.shape[1])]
    cols = [np.ascontiguousarray(c, dtype=np.float32) for c in cols]
    m = sum(c.size for c in cols)
    t0 = time.perf_counter()
    for c in cols:
        O.quantize(c)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    out["cpu_baseline"] = {"value": round(m / cpu_ms / 1e3, 3), "unit": "Mvalues/s (quantize)", "cores": 1,
                           "kind": "port", "sample": f"the grid and 3 sh0 columns ({m} of {n} values), "
                                                     f"{cpu_ms / 1e3:.1f} s; C oracle of io.py:123-167"}
    return out


def oracle_view_step(scene, cam, threads):
    """preprocess + binning + forward + backward of one view on the CPU oracle."""
    from oracle import oracle as O
    O.set_threads(threads)
    nd, bb, bits = O.preprocess(cam, scene.vox_center, scene.vox_size, scene.is_leaf)
    keys, vals, ranges = O.binning(cam, scene.octpath, nd, bb, bits)
    vis = np.where(nd > 0)[0]
    geos = O.gather_geo(vis, scene.vox_key, scene.geo_grid_pts, scene.n_vox)
    rgbs = O.sh_eval(3, vis, scene.vox_center, cam.position, scene.sh0, scene.shs)
    f = O.render_fwd(cam, np.zeros(3, np.float32), 3, True, True, ranges, vals, bb, scene.vox_center, scene.vox_size,
                     geos, rgbs, scene.s_val)
    rng = np.random.default_rng(0)
    Hc, Wc = cam.height, cam.width
    g = [rng.normal(size=s).astype(np.float32) for s in ((3, Hc, Wc), (4, Hc, Wc), (3, Hc, Wc))]
    O.render_bwd(cam, np.zeros(3, np.float32), True, True, ranges, f["tile_last"], vals, bb, scene.vox_center,
                 scene.vox_size, geos, rgbs, scene.s_val, f["T"], f["n_contrib"], g[0], g[1], g[2],
                 np.zeros((1, Hc, Wc), np.float32))
    return Hc * Wc


def run_full(args):
    """The full reconstruction workload on one GPU: the training step over 128 views of
    1024x768 (graph-captured; the views rendered 32 at a time, their gradients summed before
    Adam), then the extraction: the median depth and transmittance of 200 views rendered in
    two batches and fused into every grid point (FP64 running sums, truncation 3 finest
    voxels), and marching cubes over the level-12 voxels of the fused field.  CUDA events."""
    import torch
    from svraster_b200 import _lib
    from svraster_b200 import synthetic as S
    from svraster_b200._lib import check, ptr, stream_ptr
    from svraster_b200.marching_cubes import torch_marching_cubes_grid
    from svraster_b200.raster import RasterState
    from svraster_b200.step import BatchedTrainStep
    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    scene, cams = make_workload(0, None, "full")
    gen_s = time.perf_counter() - t0
    step = BatchedTrainStep(scene, cams, device=dev, lambda_R_concen=0.1, view_chunk=args.view_chunk)
    L = _lib.load()
    for _ in range(args.warmup):
        step.step()
    torch.cuda.synchronize()
    per_step = step.capture()
    for _ in range(args.warmup):
        step.replay()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(args.steps):
            step.replay()
        ev1.record()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    st_raster, st_misc = step.graph_status()
    if st_raster or st_misc:
        raise RuntimeError(f"graph replay status raster={st_raster} misc={st_misc}")
    rays = step.rays
    records = [int(c) for c in step.capacity]
    step.step(time_render=True)
    torch.cuda.synchronize()
    stages = {k: round(v, 3) for k, v in BatchedTrainStep.stage_ms(step.ev).items()}
    grid, centers, lengths, octpath, is_leaf = step.grid, step.centers, step.lengths, step.octpath, step.is_leaf
    geos, s_val = step.geos, step.s_val
    step.graph = None
    del step
    torch.cuda.empty_cache()
    # ---------------------------------------------------------------- extraction
    tcams = S.room_cameras(200, 1024, 768, seed=1)
    xyz = torch.as_tensor(scene.grid_pts_xyz).to(dev).contiguous()
    M = xyz.shape[0]
    h = scene.scene_extent * 2.0 ** -int(scene.octlevel.max())
    wacc = torch.zeros(M, dtype=torch.float64, device=dev)
    sacc = torch.zeros(M, dtype=torch.float64, device=dev)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)

    def view_dicts(cs):
        return [dict(width=c.width, height=c.height, tanfovx=c.tanfovx, tanfovy=c.tanfovy, cx=c.cx, cy=c.cy,
                     near=c.near, w2c=t(c.w2c), c2w=t(c.c2w), bg=torch.zeros(3, device=dev)) for c in cs]
    rgb0 = torch.zeros(100 * scene.n_vox, 3, device=dev)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    render_ms = fuse_ms = 0.0
    for a in range(0, len(tcams), 100):
        vc = tcams[a:a + 100]
        views = view_dicts(vc)
        e[0].record()
        st_ = RasterState(views, scene.n_vox, dev)
        st_.preprocess(octpath, centers, lengths, is_leaf)
        st_.bin(octpath)
        _, depth, _, T, _ = st_.render(3, True, False, centers, lengths, geos, rgb0[:len(vc) * scene.n_vox], s_val,
                                       rgb_per_view=True)
        e[1].record()
        proj = []
        for c in vc:
            proj += [c.tanfovx, c.tanfovy, 0.5, 0.5]
        proj_h = (len(proj) * _lib.C.c_double)(*proj)
        check(L.svr_tsdf_integrate(st_.views, proj_h, len(vc), M, ptr(xyz), ptr(depth), 4, 2, ptr(T), 1, 0, 1, None,
                                   3.0 * h, 0.01, 0.5, 1, 0, 0, 10.0, 1, ptr(wacc), ptr(sacc), stream_ptr(dev)),
              "tsdf")
        e[2].record()
        torch.cuda.synchronize()
        render_ms += e[0].elapsed_time(e[1])
        fuse_ms += e[1].elapsed_time(e[2])
        del st_, depth, T
    tsdf = torch.where(wacc > 0, sacc / wacc, torch.full_like(wacc, float("nan"))).float()
    lv12 = torch.as_tensor(scene.octlevel.reshape(-1) == int(scene.octlevel.max())).to(dev)
    key12 = torch.as_tensor(scene.vox_key).to(dev)[lv12].contiguous()
    torch_marching_cubes_grid(tsdf, xyz, key12[:1024], 0.0)   # warm up
    e[0].record()
    verts, faces = torch_marching_cubes_grid(tsdf, xyz, key12, 0.0)
    e[1].record()
    torch.cuda.synchronize()
    mc_ms = e[0].elapsed_time(e[1])
    n_faces, n_verts = int(faces.shape[0]), int(verts.shape[0])
    fused = int((wacc > 0).sum().item())
    del tsdf, wacc, sacc, verts, faces
    torch.cuda.empty_cache()
    # the reference's own extension per view on a sample of the training views (its whole
    # step over all 128 views would take minutes): rays per second of its per-view step
    ref = {"unavailable": "skipped (--no-per-view)"}
    if not args.no_per_view:
        ref = run_reference_cuda(scene, cams[:8], dev, steps=2, warmup=1)
        if "value" in ref:
            ref["sample"] = "the first 8 of the 128 training views"
    out = {"metric": "fwd+bwd Mrays/s", "value": round(rays / ms / 1e3, 3), "unit": "Mrays/s",
            "ms_per_step": round(ms, 3), "iters_per_s": round(1e3 / ms, 3), "steps": args.steps,
            "config": {"workload": CONFIGS["full"]["workload"], "n_voxels": scene.n_vox, "n_grid_pts": M,
                       "views": len(cams), "view_chunk": args.view_chunk, "rays_per_step": rays,
                       "records_per_chunk": records, "scene_generation_s": round(gen_s, 1)},
            "stages_ms_eager": stages, "kernels_per_step": per_step, "clocks": clk.summary(),
            "extraction": {"views": len(tcams), "render_ms": round(render_ms, 3), "tsdf_fp64_ms": round(fuse_ms, 3),
                           "fused_points": fused, "grid_points": M,
                           "mc_level": int(scene.octlevel.max()), "mc_voxels": int(lv12.sum().item()),
                           "mc_ms": round(mc_ms, 3), "mc_faces": n_faces, "mc_verts": n_verts},
           "reference_cuda": ref}
    if "value" in ref:
        out["vs_reference_cuda"] = {"value": round(out["value"] / ref["value"], 3)}
    return out


def sample_views(cams):
    """The CPU sample of a workload: the first view of each distinct resolution, in order."""
    seen, out = set(), []
    for c in cams:
        if (c.width, c.height) not in seen:
            seen.add((c.width, c.height))
            out.append(c)
    return out


def cpu_baseline(scene, cams):
    views = sample_views(cams)
    t0 = time.perf_counter()
    rays = sum(oracle_view_step(scene, c, threads=1) for c in views)
    dt = time.perf_counter() - t0
    sizes = ", ".join(f"{c.width}x{c.height}" for c in views)
    return {"value": round(rays / dt / 1e6, 5), "unit": "Mrays/s", "cores": 1, "kind": "port",
            "sample": f"{len(views)} of {len(cams)} views ({sizes}) preprocess+binning+fwd+bwd, "
                      f"single thread, {dt:.1f} s"}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args):
    config = getattr(args, "config", DEFAULT_CONFIG)
    scene, cams = make_workload(0, config=config)
    views = sample_views(cams)
    threads = os.cpu_count() or 1
    oracle_view_step(scene, views[0], threads)  # warm caches / page in
    for i in range(max(0, args.warmup - 1)):
        oracle_view_step(scene, views[(i + 1) % len(views)], threads)
    times, rays = [], 0
    for i in range(args.steps):
        t0 = time.perf_counter()
        rays_i = oracle_view_step(scene, views[i % len(views)], threads)
        times.append(time.perf_counter() - t0)
        rays += rays_i
    total = sum(times)
    value = rays / total / 1e6
    sizes = ", ".join(f"{c.width}x{c.height}" for c in views)
    return {"metric": "fwd+bwd Mrays/s", "value": round(value, 5), "unit": "Mrays/s", "impl": "reference",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": CONFIGS[config]["workload"], "n_voxels": scene.n_vox,
                       "sample": f"one view per step, rotating over the workload's resolutions ({sizes}); "
                                 "preprocess+binning+fwd+bwd"},
            "cpu_baseline": {"value": round(value, 5), "unit": "Mrays/s", "cores": threads, "kind": "port",
                             "sample": f"one view per step ({sizes}, rotating) of the {len(cams)}-view workload"},
            "e2e": {"value": round(value, 5), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def secondary_summary(res):
    """The fields of a secondary workload's line kept in the headline line."""
    keep = ("value", "unit", "ms_per_step", "iters_per_s", "config", "stages_ms", "roofline", "clocks", "cuda_graph",
            "autotuned_render", "gpu_launches")
    return {k: res[k] for k in keep if k in res}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default=DEFAULT_CONFIG, choices=sorted(CONFIGS),
                    help=f"workload ({DEFAULT_CONFIG} = the headline)")
    ap.add_argument("--views", type=int, default=None, help="views per GPU (default: the workload's)")
    ap.add_argument("--per-view-steps", type=int, default=5, help="timed steps of the per-view legs")
    ap.add_argument("--view-chunk", type=int, default=32, help="views per chunk of the full workload's step")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extract", action="store_true", help="skip the extraction / regulariser / format legs")
    ap.add_argument("--no-per-view", action="store_true", help="skip the per-view and reference-CUDA legs")
    ap.add_argument("--no-mid", action="store_true", help="skip the secondary mid-size workload")
    ap.add_argument("--no-graph", action="store_true", help="time eager steps instead of graph replays")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default render launch configuration")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return

    if args.config == "full":
        if rank == 0:
            print(json.dumps(run_full(args)), flush=True)
        return
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(dev)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    result, step, scene, cams = run_ours(args, rank, world, args.config)
    if world > 1:
        # several ranks: the headline line only (the other legs are single-GPU measurements)
        if rank == 0:
            print(json.dumps(result), flush=True)
        import torch.distributed as dist
        step.graph = step.graph_b = None   # graphs holding NCCL calls go before the group does
        del step
        dist.barrier()
        dist.destroy_process_group()
        return
    if rank == 0:
        # everything below runs after the headline's timed region
        step.graph = step.graph_b = None
        del step
        torch.cuda.empty_cache()
        if not args.no_e2e:
            result["e2e"] = run_e2e_batched(args, scene, cams, dev)
        result["native_step"] = run_native_step(args, scene, cams, dev)
        if not args.no_per_view:
            pv = run_per_view(args, scene, cams, dev, host_inputs=False, steps=args.per_view_steps)
            result["per_view"] = pv
            result["batched_vs_per_view"] = {"value": round(result["value"] / pv["value"], 3)}
            if not args.no_e2e:
                pve = run_per_view(args, scene, cams, dev, host_inputs=True, steps=args.per_view_steps)
                result["e2e_per_view"] = pve
                result["batched_vs_per_view"]["e2e"] = round(result["e2e"]["value"] / pve["value"], 3)
            result["reference_cuda"] = run_reference_cuda(scene, cams, dev)
            if "value" in result["reference_cuda"]:
                result["vs_reference_cuda"] = {"value": round(result["value"] / result["reference_cuda"]["value"], 3)}
                if "e2e" in result:
                    result["vs_reference_cuda"]["e2e"] = round(result["e2e"]["value"] /
                                                               result["reference_cuda"]["value"], 3)
        if not args.no_cpu:
            result["cpu_baseline"] = cpu_baseline(scene, cams)
        if args.config != "mid" and not args.no_mid:
            # the plain mid-size workload: its own step, e2e, per-view and reference legs, and the
            # extraction / regulariser / format legs on its scene
            margs = argparse.Namespace(**vars(args))
            margs.views = None
            mres, mstep, mscene, mcams = run_ours(margs, rank, world, "mid")
            mid = secondary_summary(mres)
            if not args.no_extract:
                mid["extraction"] = run_extraction(mstep, mscene, mcams, dev)
                mid["adaptive"] = run_adaptive(mstep, mscene, mcams, dev)
                mid["regularisers"] = run_regularisers(mstep, mscene, dev)
                mid["checkpoint"] = run_checkpoint(mscene, dev)
                mid["normal_losses"] = run_normal_losses(mstep, mcams, dev)
                mid["normal_losses"]["step_with_losses"] = run_step_with_normal_losses(mscene, mcams, dev)
            mstep.graph = mstep.graph_b = None
            del mstep
            torch.cuda.empty_cache()
            if not args.no_e2e:
                mid["e2e"] = run_e2e_batched(margs, mscene, mcams, dev)
            if not args.no_per_view:
                mid["per_view"] = run_per_view(margs, mscene, mcams, dev, host_inputs=False)
                if not args.no_e2e:
                    mid["e2e_per_view"] = run_per_view(margs, mscene, mcams, dev, host_inputs=True)
                mid["reference_cuda"] = run_reference_cuda(mscene, mcams, dev, steps=5, warmup=2)
            result["mid_size"] = mid
        print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
