"""Autotuner for the render kernels' launch variant.

The forward and adjoint tile kernels come in several compiled variants: the kernel family
(pairs numbered over the whole CTA, pairs per warp, or the per-warp filter kernels), ring
depth (shared-memory slots of 128 records) and CTAs per SM (the occupancy the register
allocator is asked to meet).  These change only the schedule: every variant produces the same
forward outputs bit for bit and the same gradients up to the order of float atomics.  Which one is fastest depends on the workload (records per tile, image sizes, how
unevenly the work falls on the tiles), so the tuner times each on the caller's own binned
batch and keeps the fastest.  Tile shape and samples per voxel are not tuned: the 16x16 tile
is part of the binning format the buffers share with the reference's, and the number of
samples per voxel (vox_geo_mode) changes the rendered model.

Results can be kept in a JSON file keyed by GPU and workload signature (``cache=``); nothing is
written unless a path is given.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import torch

from . import _lib
from ._lib import check


def configs():
    """{"fwd": [(index, impl, ring, ctas_per_sm), ...], "bwd": [...]}"""
    L = _lib.load()
    nf, nb = C.c_int(0), C.c_int(0)
    check(L.svr_render_config_count(C.byref(nf), C.byref(nb)), "config count")
    out = {}
    for name, pass_id, n in (("fwd", 0, nf.value), ("bwd", 1, nb.value)):
        rows = []
        for i in range(n):
            impl, ring, ctas = C.c_int(0), C.c_int(0), C.c_int(0)
            check(L.svr_render_config_describe(pass_id, i, C.byref(impl), C.byref(ring), C.byref(ctas)),
                  "config describe")
            rows.append((i, impl.value, ring.value, ctas.value))
        out[name] = rows
    return out


def _label(impl, ring, ctas):
    return f"impl{impl}_ring{ring}_cta{ctas}"


def get_config():
    f, b = C.c_int(0), C.c_int(0)
    check(_lib.load().svr_render_get_config(C.byref(f), C.byref(b)), "get config")
    return f.value, b.value


def set_config(fwd_index, bwd_index):
    check(_lib.load().svr_render_set_config(int(fwd_index), int(bwd_index)), "set config")


def _time(fn, reps):
    fn()                                  # first launch of a configuration sets it up
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    times = []
    for _ in range(reps):
        ev[0].record()
        fn()
        ev[1].record()
        torch.cuda.synchronize()
        times.append(ev[0].elapsed_time(ev[1]))
    times.sort()
    return times[len(times) // 2]


def tune_render(run_fwd, run_bwd, reps=3, key=None, cache=None):
    """Time every forward configuration with ``run_fwd()`` and every adjoint configuration with
    ``run_bwd()`` (each issues one launch on the current stream and must be repeatable), select
    the fastest of each and return {"fwd": ..., "bwd": ..., "ms": {...}}.  With ``cache`` (a
    JSON path) and ``key``, a stored choice is reused and a new one stored."""
    if cache and key and os.path.exists(cache):
        with open(cache) as f:
            stored = json.load(f).get(key)
        if stored:
            set_config(stored["fwd"], stored["bwd"])
            return dict(stored, cached=True)
    cfg = configs()
    f0, b0 = get_config()
    ms_f, ms_b = {}, {}
    for i, impl, ring, ctas in cfg["fwd"]:
        set_config(i, b0)
        ms_f[_label(impl, ring, ctas)] = (i, _time(run_fwd, reps))
    f_ms = {i: t for i, t in ms_f.values()}
    best_f = min(f_ms, key=f_ms.get)
    # The CTA-wide adjoint (family 3) reads the candidate rows its forward (family 3) wrote and
    # otherwise filters again, so the adjoint variants are timed after one run of the forward
    # they will follow; when the fastest forward alone is of another family, the fastest
    # family-3 forward is tried with them too and the pair with the lower total kept.
    fam3 = [i for i, impl, _, _ in cfg["fwd"] if impl == 3]
    cands = [best_f] + ([min(fam3, key=f_ms.get)] if fam3 and best_f not in fam3 else [])
    best = None
    for f in cands:
        set_config(f, b0)
        run_fwd()
        ms_f_b = {}
        for i, impl, ring, ctas in cfg["bwd"]:
            set_config(f, i)
            ms_f_b[_label(impl, ring, ctas)] = (i, _time(run_bwd, reps))
        b_i, b_t = min(ms_f_b.values(), key=lambda t: t[1])
        if best is None or f_ms[f] + b_t < best[0]:
            best = (f_ms[f] + b_t, f, b_i, ms_f_b)
    _, best_f, best_b, ms_b = best
    set_config(best_f, best_b)
    res = {"fwd": best_f, "bwd": best_b,
           "fwd_config": dict(zip(("impl", "ring", "ctas_per_sm"), cfg["fwd"][best_f][1:])),
           "bwd_config": dict(zip(("impl", "ring", "ctas_per_sm"), cfg["bwd"][best_b][1:])),
           "ms": {"fwd": {k: round(v[1], 4) for k, v in ms_f.items()},
                  "bwd": {k: round(v[1], 4) for k, v in ms_b.items()}}}
    if cache and key:
        data = {}
        if os.path.exists(cache):
            with open(cache) as f:
                data = json.load(f)
        data[key] = {k: res[k] for k in ("fwd", "bwd", "fwd_config", "bwd_config")}
        os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
        with open(cache, "w") as f:
            json.dump(data, f, indent=1)
    return res


def workload_key(device, n_views, total_pixels, n_vox, records):
    """GPU name and a coarse workload signature (records rounded to 2 significant digits)."""
    r = int(float(f"{records:.2g}"))
    return f"{torch.cuda.get_device_name(device)}|views={n_views}|pixels={total_pixels}|voxels={n_vox}|records~{r}"
