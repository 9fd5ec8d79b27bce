"""The oracle's normal-from-depth consistency losses against the reference's own torch code
(tests/golden/nd_*.npz, made by tests/golden/make_golden_nd.py): loss values and the autograd
gradients with respect to the depth planes and the rendered normals."""
from __future__ import annotations

import os

import numpy as np
import pytest

from tests.golden.nd_cases import ND_CASES, nd_camera, nd_inputs

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# reference float32 torch ops (norm reductions, unfused cross products) vs the oracle's float32
# expressions: gradients agree to a few 1e-6 of their largest entry
LOSS_RTOL, GRAD_TOL = 1e-5, 2e-5


def oracle_case(name, case, g):
    from oracle import oracle as O
    cam = nd_camera(case)
    depth, normal, T = nd_inputs(case, g["c2w"])
    if case["mode"] == "dmean":
        tol = float(np.float32(np.cos(np.deg2rad(case["tol_deg"]))))
        plane, Tp, ks = 0, T[0], case["ks"]
    else:
        tol, plane, Tp, ks = -1.0, 2, None, 3
    loss, gd, gn = O.normal_depth_loss(case["W"], case["H"], cam.cx, cam.cy, cam.tanfovx, cam.tanfovy, g["c2w"],
                                       depth[plane], normal, Tp, ks, tol)
    full = np.zeros_like(depth)
    full[plane] = gd
    return loss, full, gn


@pytest.mark.parametrize("name", list(ND_CASES))
def test_oracle_matches_reference_losses(name):
    g = np.load(os.path.join(HERE, f"nd_{name}.npz"))
    loss, gd, gn = oracle_case(name, ND_CASES[name], g)
    assert abs(loss - float(g["loss"])) <= LOSS_RTOL * abs(float(g["loss"]))
    assert np.abs(gd - g["grad_depth"]).max() <= GRAD_TOL * np.abs(g["grad_depth"]).max()
    assert np.abs(gn - g["grad_normal"]).max() <= GRAD_TOL * np.abs(g["grad_normal"]).max()
    # the reference's gradient reaches only the plane the loss reads
    other = [p for p in range(4) if p != (0 if ND_CASES[name]["mode"] == "dmean" else 2)]
    assert not g["grad_depth"][other].any()
