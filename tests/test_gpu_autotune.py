"""Every compiled launch variant of the render kernels (kernel family x ring slots x CTAs per
SM) gives the same results, and the autotuner picks one of them and leaves it in force."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from svraster_b200 import autotune as AT
from svraster_b200 import synthetic as S
from svraster_b200.step import BatchedTrainStep

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def step():
    sc = S.scene_small(seed=3)
    cams = S.fibonacci_cameras(3, 3.0, 160, 120, fovx_deg=50.0)
    st = BatchedTrainStep(sc, cams, device="cuda", lambda_R_concen=0.1)
    st.step()
    yield st
    AT.set_config(0, 0)


def _fwd(st):
    color, depth, normal, T, _ = st.state.render(3, True, True, st.centers, st.lengths, st.geos, st.rgbs, st.s_val,
                                                 rgb_per_view=True)
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in (color, depth, normal, T)], T


def _bwd(st, T):
    st.dvox.zero_(); st.drgbs.zero_(); st.ds.zero_()
    st.state.render_backward(True, True, st.s_val, T, st.dcolor, st.ddepth, st.dnormal, st.dT,
                             lambda_R_concen=st.lambda_R, gt_color=st.gt, drgbs=st.drgbs, dvox=st.dvox, ds=st.ds)
    torch.cuda.synchronize()
    return st.dvox.cpu().numpy().copy(), st.drgbs.cpu().numpy().copy(), float(st.ds.item())


def test_all_configurations_agree(step):
    cfg = AT.configs()
    assert len(cfg["fwd"]) >= 2 and len(cfg["bwd"]) >= 2
    AT.set_config(0, 0)
    ref, T = _fwd(step)
    dv0, dr0, ds0 = _bwd(step, T)
    for i, *_ in cfg["fwd"]:
        AT.set_config(i, 0)
        out, _ = _fwd(step)
        for a, b in zip(out, ref):
            assert np.array_equal(a, b), f"forward configuration {i} differs"
    for j, *_ in cfg["bwd"]:
        AT.set_config(0, j)
        dv, dr, ds = _bwd(step, T)
        # float atomics: summation order only
        np.testing.assert_allclose(dv, dv0, rtol=1e-4, atol=1e-4 * np.abs(dv0).max())
        np.testing.assert_allclose(dr, dr0, rtol=1e-4, atol=1e-4 * np.abs(dr0).max())
        assert abs(ds - ds0) <= 1e-4 * abs(ds0) + 1e-6
    assert step.state.status() == 0


def test_autotune_selects_and_applies(step, tmp_path):
    cache = str(tmp_path / "tune.json")
    res = step.autotune(reps=2, cache=cache)
    assert AT.get_config() == (res["fwd"], res["bwd"])
    assert set(res["ms"]["fwd"]) and set(res["ms"]["bwd"])
    again = step.autotune(reps=2, cache=cache)
    assert again.get("cached") and (again["fwd"], again["bwd"]) == (res["fwd"], res["bwd"])
