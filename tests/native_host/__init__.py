"""Build and feed ``step_driver.c``, the plain-C host of the batched step (svr_step_*)."""
from __future__ import annotations

import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIBDIR = os.path.join(ROOT, "svraster_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def compile_driver(out_dir):
    """gcc -std=c11 -Wall -Werror against the public header, linked to the in-tree library and
    the CUDA runtime.  Returns the binary's path."""
    exe = os.path.join(out_dir, "step_driver")
    cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(HERE, "step_driver.c"), "-o", exe,
           "-L", LIBDIR, "-lsvraster_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"step_driver build failed:\n{r.stdout}\n{r.stderr}")
    return exe


def layout(exe):
    r = subprocess.run([exe, "--layout"], capture_output=True, text=True, check=True)
    return {k: int(v) for k, v in (line.split() for line in r.stdout.splitlines())}


def write_input(path, scene, cams, upstream, hyper):
    """The driver's input file (format in step_driver.c).  ``upstream`` = (dcolor, ddepth,
    dnormal) float32 arrays of 3P, 4P, 3P; ``hyper`` a dict of the header's scalars."""
    deg = hyper["sh_degree"]
    M = (deg + 1) ** 2
    N = int(scene.n_vox)
    grid = np.ascontiguousarray(scene.geo_grid_pts, np.float32).reshape(-1)
    head = np.array([N, grid.size, deg, len(cams), hyper["grid_res_pow2"], hyper["seed"], scene.scene_extent,
                     scene.s_val, hyper["lambda_ls"], hyper["lambda_ge"], *hyper["lr"], *hyper["betas"],
                     hyper["eps"]], np.float64)
    assert head.size == 16
    with open(path, "wb") as f:
        f.write(head.tobytes())
        f.write(np.ascontiguousarray(scene.octpath, np.int64).tobytes())
        f.write(np.ascontiguousarray(scene.vox_center, np.float32).tobytes())
        f.write(np.ascontiguousarray(scene.vox_size, np.float32).reshape(-1).tobytes())
        f.write(np.ascontiguousarray(scene.is_leaf, np.uint8).reshape(-1).tobytes())
        f.write(np.ascontiguousarray(scene.vox_key, np.int64).tobytes())
        f.write(grid.tobytes())
        f.write(np.ascontiguousarray(scene.sh0, np.float32).tobytes())
        shs = np.ascontiguousarray(scene.shs, np.float32)
        assert shs.size == N * (M - 1) * 3
        f.write(shs.tobytes())
        for c in cams:
            f.write(np.array([c.width, c.height], np.int32).tobytes())
            f.write(np.array([c.tanfovx, c.tanfovy, c.cx, c.cy, c.near], np.float32).tobytes())
            f.write(np.ascontiguousarray(c.w2c, np.float32).tobytes())
            f.write(np.ascontiguousarray(c.c2w, np.float32).tobytes())
        for a in upstream:
            f.write(np.ascontiguousarray(a, np.float32).tobytes())


def read_output(path, P, n_grid, N, M):
    buf = open(path, "rb").read()
    info = np.frombuffer(buf, np.int64, 8, 0)
    status = np.frombuffer(buf, np.uint32, 2, 64)
    off = 72
    out = {"info": info, "status": status}
    for name, n in (("color", 3 * P), ("T", P), ("grad_flat", int(info[4])), ("grid", n_grid), ("sh0", 3 * N),
                    ("shs", 3 * N * (M - 1))):
        out[name] = np.frombuffer(buf, np.float32, n, off)
        off += 4 * n
    assert off == len(buf)
    return out
