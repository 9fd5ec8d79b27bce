"""Golden vectors for the normal-from-depth consistency losses from the reference's own code.

Executes src/cameras.py and src/utils/loss_utils.py of the reference in place on the CPU
("cuda" device strings mapped to "cpu"; nothing is copied into this repository; the image
metrics that loss_utils imports at the top, lpips / pytorch_msssim / fused_ssim, are absent
here and stubbed, the losses used do not call them).  For each case of ``nd_cases.ND_CASES``
runs NormalDepthConsistencyLoss (loss_utils.py:345-379) or NormalMedianConsistencyLoss
(loss_utils.py:381-407) with autograd and writes tests/golden/nd_<case>.npz: the reference
camera's c2w (its float32 inverse of w2c), the loss, and the gradients with respect to the
depth planes and the rendered normals.

Usage (this machine, with the reference sources):
    python tests/golden/make_golden_nd.py [/path/to/reference]
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests.golden.nd_cases import ND_CASES, nd_camera, nd_inputs  # noqa: E402
from tests.golden.make_golden_extract import load_on_cpu  # noqa: E402


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SVR_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: give the reference checkout as the first argument or in SVR_REFERENCE_DIR")
    import svraster_b200
    svraster_b200.install_as_svraster_cuda()   # cameras.py calls svraster_cuda.utils.compute_rd
    for name, attr in (("lpips", "LPIPS"), ("pytorch_msssim", "SSIM"), ("fused_ssim", "fused_ssim")):
        m = types.ModuleType(name)
        setattr(m, attr, None)
        sys.modules[name] = m
    cams_mod = load_on_cpu(os.path.join(ref, "src", "cameras.py"), "ref_cameras")
    loss_mod = load_on_cpu(os.path.join(ref, "src", "utils", "loss_utils.py"), "ref_loss_utils")
    here = os.path.dirname(os.path.abspath(__file__))
    for name, case in ND_CASES.items():
        cam = nd_camera(case)
        rcam = cams_mod.Camera("v", cam.w2c.astype(np.float64), cam.fovx, cam.fovy, 0.5, 0.5, near=0.02,
                               image=torch.zeros(3, case["H"], case["W"]))
        c2w = rcam.c2w.numpy().astype(np.float32)
        depth, normal, T = nd_inputs(case, c2w)
        d = torch.from_numpy(depth).requires_grad_()
        n = torch.from_numpy(normal).requires_grad_()
        pkg = {"raw_depth": d, "raw_normal": n, "raw_T": torch.from_numpy(T)}
        if case["mode"] == "dmean":
            fn = loss_mod.NormalDepthConsistencyLoss(iter_from=0, iter_end=10, ks=case["ks"], tol_deg=case["tol_deg"])
        else:
            fn = loss_mod.NormalMedianConsistencyLoss(iter_from=0, iter_end=10)
        loss = fn(rcam, pkg, 5)
        loss.backward()
        np.savez_compressed(os.path.join(here, f"nd_{name}.npz"), c2w=c2w, loss=np.float32(loss.item()),
                            grad_depth=d.grad.numpy(), grad_normal=n.grad.numpy())
        print(name, float(loss), float(d.grad.abs().max()), float(n.grad.abs().max()))


if __name__ == "__main__":
    main()
