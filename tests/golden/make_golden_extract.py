"""Golden vectors for TSDF fusion and marching cubes from the reference's own torch code.

The reference implements both in torch (src/utils/fuser_utils.py, src/cameras.py,
cuda/svraster_cuda/marching_cubes.py).  This script executes those files in place on the
CPU through a loader that maps their "cuda" device strings to "cpu" (nothing is copied
into this repository) and writes tests/golden/extract_*.npz.  Inputs are seeded synthetic
scenes; the depth / transmittance maps fused here come from the C oracle's renderer.

Usage (this machine, with the reference sources):
    python tests/golden/make_golden_extract.py [/path/to/reference] [--only CASE ...]
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests.golden.extract_cases import TSDF_CASES, MC_CASES, tsdf_inputs, mc_inputs, mesh_digest  # noqa: E402


def load_on_cpu(path, name, extra=None):
    src = open(path).read().replace('device="cuda"', 'device="cpu"').replace(".cuda()", ".cpu()")
    mod = types.ModuleType(name)
    mod.__file__ = path
    if extra:
        mod.__dict__.update(extra)
    exec(compile(src, path, "exec"), mod.__dict__)
    return mod


def main():
    args = sys.argv[1:]
    only = set(args[args.index("--only") + 1:]) if "--only" in args else None
    if "--only" in args:
        args = args[:args.index("--only")]
    ref = args[0] if args else os.environ.get("SVR_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: give the reference checkout as the first argument or in SVR_REFERENCE_DIR")
    import svraster_b200
    svraster_b200.install_as_svraster_cuda()   # cameras.py imports svraster_cuda (unused here)
    cams_mod = load_on_cpu(os.path.join(ref, "src", "cameras.py"), "ref_cameras")
    fuser_mod = load_on_cpu(os.path.join(ref, "src", "utils", "fuser_utils.py"), "ref_fuser")
    mc_mod = load_on_cpu(os.path.join(ref, "cuda", "svraster_cuda", "marching_cubes.py"), "ref_mc")
    out_dir = os.path.dirname(os.path.abspath(__file__))

    for name, case in TSDF_CASES.items():
        if only is not None and name not in only:
            continue
        inp = tsdf_inputs(case)
        cams = []
        for c in inp["cams"]:
            cams.append(cams_mod.Camera("v", c.w2c.astype(np.float64), c.fovx, c.fovy, 0.5, 0.5, near=0.02,
                                        image=torch.zeros(3, c.height, c.width)))
        bw = inp["bandwidth"]
        bandwidth = torch.from_numpy(bw) if isinstance(bw, np.ndarray) else bw
        fuser = fuser_mod.Fuser(xyz=torch.from_numpy(inp["xyz"]), bandwidth=bandwidth, use_trunc=case["use_trunc"],
                                fuse_tsdf=True, feat_dim=0, alpha_thres=case["alpha_thres"],
                                crop_border=case["crop_border"], normal_weight=False,
                                depth_weight=case["depth_weight"], border_weight=case["border_weight"],
                                use_half=False)
        for cam, d, a in zip(cams, inp["depths"], inp["alphas"]):
            fuser.integrate(cam, torch.from_numpy(d), alpha=torch.from_numpy(a))
        np.savez_compressed(os.path.join(out_dir, f"extract_{name}.npz"), digest=inp["digest"],
                            c2w=np.stack([c.c2w.numpy() for c in cams]), w2c=np.stack([c.w2c.numpy() for c in cams]),
                            tanfov=np.array([[c.tanfovx, c.tanfovy] for c in cams]),
                            weight=fuser.weight.numpy(), sd_val=fuser.sd_val.numpy(), tsdf=fuser.tsdf.numpy())
        print(name, "fused points", int((fuser.weight > 0).sum()))

    for name, case in MC_CASES.items():
        if only is not None and name not in only:
            continue
        inp = mc_inputs(case)
        verts, faces = mc_mod.torch_marching_cubes_grid(torch.from_numpy(inp["val"]), torch.from_numpy(inp["xyz"]),
                                                        torch.from_numpy(inp["vox_key"]), case["iso"])
        if case.get("compact"):
            np.savez_compressed(os.path.join(out_dir, f"extract_{name}.npz"), digest=inp["digest"],
                                **mesh_digest(verts.numpy(), faces.numpy()))
        else:
            np.savez_compressed(os.path.join(out_dir, f"extract_{name}.npz"), digest=inp["digest"],
                                verts=verts.numpy(), faces=faces.numpy())
        print(name, "verts", len(verts), "faces", len(faces))


if __name__ == "__main__":
    main()
