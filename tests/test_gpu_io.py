"""Checkpoint formats on the GPU: the library's 8-bit codebook (``svr_quantize``) against the
C oracle (pinned bit for bit to the reference's quantization()), and save / load through
``svraster_b200.io`` against checkpoints written by the reference's SVInOut.save."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from svraster_b200 import adaptive as A
from svraster_b200 import io
from svraster_b200.sparse_adam import SparseAdam
from tests.golden.io_cases import QUANT_CASES, model_fields, quant_values, small_scene

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def check_codebook(got_idx, got_book, vals, ref_idx, ref_book, rtol=1e-5, atol=1e-7):
    """The library sums each entry's mean in float64, the reference (and the oracle) in float32
    in value order, whose rounding grows with the entry's population: codebooks agree to
    ``rtol`` plus ``atol`` times the largest entry (1e-5 / 1e-7 for entries of up to a few
    hundred values, 1e-4 / 1e-6 for 16k, where an entry near zero keeps the absolute
    rounding of its running sum), indices except for values at a near-tie between two
    entries, and the mean reconstruction error to ``rtol``."""
    same = got_idx == ref_idx
    assert same.mean() >= 0.999, f"index agreement {same.mean():.5f}"
    used = np.bincount(ref_idx.reshape(-1), minlength=256) > 0
    np.testing.assert_allclose(got_book[used], ref_book[used], rtol=rtol, atol=atol * np.abs(ref_book).max())
    e_got = np.abs(got_book[got_idx] - vals).mean()
    e_ref = np.abs(ref_book[ref_idx] - vals).mean()
    assert abs(e_got - e_ref) <= rtol * max(e_ref, 1e-30) + 1e-12


@pytest.mark.parametrize("name", QUANT_CASES)
def test_codebook_matches_oracle(name):
    from oracle import oracle as O
    vals = quant_values(name)
    q = io.quantization(torch.from_numpy(vals).cuda())
    idx, book = q["index"].cpu().numpy(), q["codebook"].cpu().numpy()
    ref_idx, ref_book, _ = O.quantize(vals)
    assert idx.shape == vals.shape and idx.dtype == np.uint8
    check_codebook(idx, book, vals, ref_idx, ref_book)
    if name in ("small", "one"):          # no rounds: a pure function of the quantiles
        assert np.array_equal(idx, ref_idx)


def test_codebook_at_scale_matches_oracle():
    """4M values (one SH column of a mid-size model), the bench's sizes."""
    from oracle import oracle as O
    vals = (0.2 * np.random.default_rng(9).standard_t(5, size=1 << 22)).astype(np.float32)
    q = io.quantization(torch.from_numpy(vals).cuda())
    ref_idx, ref_book, _ = O.quantize(vals)
    check_codebook(q["index"].cpu().numpy(), q["codebook"].cpu().numpy(), vals, ref_idx, ref_book, rtol=1e-4,
                   atol=1e-6)


def test_dequantization_is_codebook_lookup():
    rng = np.random.default_rng(3)
    idx = rng.integers(0, 256, size=(1000, 1, 3)).astype(np.uint8)
    book = rng.normal(size=256).astype(np.float32)
    out = io.dequantization({"index": torch.from_numpy(idx).cuda(), "codebook": torch.from_numpy(book).cuda()})
    assert np.array_equal(out.cpu().numpy(), book[idx])


class _Model(io.SVInOut, io.SVOptimizerIO):
    pass


def _check_loaded(m, fields, sd_values):
    sc = small_scene()
    for k in ("scene_center", "inside_extent", "scene_extent", "octpath", "octlevel", "_log_s", "is_leaf"):
        assert np.array_equal(getattr(m, k).detach().cpu().numpy(), fields[k]), k
    for k in ("_geo_grid_pts", "_sh0", "_shs"):
        assert np.array_equal(getattr(m, k).detach().cpu().numpy(), sd_values[k]), k
    assert m.active_sh_degree == fields["active_sh_degree"] and m.ss == fields["ss"]
    cen, size = A.octpath_decoding(m.octpath, m.octlevel, m.scene_center, m.scene_extent)
    assert torch.equal(cen, m.vox_center) and torch.equal(size, m.vox_size)
    np.testing.assert_allclose(m.vox_center.cpu().numpy(), sc.vox_center, rtol=0, atol=1e-6)
    # the rebuilt link orders the grid points as the file's grid values are stored
    geo = m._geo_grid_pts.detach().cpu().numpy().reshape(-1)
    assert np.array_equal(geo[m.vox_key.cpu().numpy()], geo[sc.vox_key])
    assert m._subdiv_p.shape == (sc.n_vox, 1) and bool((m._subdiv_p == 1).all())
    assert m._geo_grid_pts.requires_grad and m._shs.requires_grad


def test_load_reference_checkpoint():
    f = model_fields()
    m = _Model()
    m.load(os.path.join(HERE, "ref_ckpt.pt"))
    _check_loaded(m, f, f)


def test_load_reference_quantized_checkpoint():
    f = model_fields()
    raw = torch.load(os.path.join(HERE, "ref_ckpt_q.pt"), map_location="cpu", weights_only=True)
    look = lambda q: q["codebook"].numpy()[q["index"].numpy().astype(np.int64)]
    deq = {"_geo_grid_pts": look(raw["_geo_grid_pts"]),
           "_sh0": np.concatenate([look(q) for q in raw["_sh0"]], axis=1),
           "_shs": np.concatenate([look(q) for q in raw["_shs"]], axis=1)}
    m = _Model()
    m.load(os.path.join(HERE, "ref_ckpt_q.pt"))
    _check_loaded(m, f, deq)


def test_save_is_the_reference_layout_and_round_trips(tmp_path):
    f = model_fields()
    m = _Model()
    m.load(os.path.join(HERE, "ref_ckpt.pt"))
    ref_plain = torch.load(os.path.join(HERE, "ref_ckpt.pt"), map_location="cpu", weights_only=True)
    ref_q = torch.load(os.path.join(HERE, "ref_ckpt_q.pt"), map_location="cpu", weights_only=True)
    m.model_path = str(tmp_path)
    m.save_iteration(7)
    m.save_iteration(12, quantize=True)
    plain = torch.load(tmp_path / "checkpoints" / "iter000007_model.pt", map_location="cpu", weights_only=True)
    assert set(plain) == set(ref_plain)
    for k, v in ref_plain.items():
        if torch.is_tensor(v):
            assert plain[k].dtype == v.dtype and torch.equal(plain[k], v), k
        else:
            assert plain[k] == v, k
    q = torch.load(tmp_path / "checkpoints" / "iter000012_model.pt", map_location="cpu", weights_only=True)
    assert set(q) == set(ref_q) and q["quantized"] is True
    assert len(q["_sh0"]) == len(ref_q["_sh0"]) and len(q["_shs"]) == len(ref_q["_shs"])
    pieces = [(q["_geo_grid_pts"], ref_q["_geo_grid_pts"], f["_geo_grid_pts"])]
    pieces += [(a, b, f["_sh0"][:, j:j + 1]) for j, (a, b) in enumerate(zip(q["_sh0"], ref_q["_sh0"]))]
    pieces += [(a, b, f["_shs"][:, j:j + 1]) for j, (a, b) in enumerate(zip(q["_shs"], ref_q["_shs"]))]
    for a, b, vals in pieces:
        assert a["index"].dtype == torch.uint8 and a["index"].shape == b["index"].shape
        check_codebook(a["index"].numpy(), a["codebook"].numpy(), vals, b["index"].numpy(), b["codebook"].numpy())
    # latest iteration is found, and the quantized file loads back to its codebook values
    m2 = _Model()
    m2.model_path = str(tmp_path)
    assert m2.load_iteration(-1) == 12
    look = lambda d: d["codebook"].numpy()[d["index"].numpy().astype(np.int64)]
    assert np.array_equal(m2._geo_grid_pts.detach().cpu().numpy(), look(q["_geo_grid_pts"]))


def test_optimizer_checkpoint_round_trip(tmp_path):
    m = _Model()
    m.load(os.path.join(HERE, "ref_ckpt.pt"))
    m.model_path = str(tmp_path)
    m.optimizer = SparseAdam([{"params": [m._geo_grid_pts], "lr": 0.01, "name": "_geo_grid_pts"},
                              {"params": [m._sh0], "lr": 0.01, "name": "_sh0"}], betas=(0.1, 0.99))
    for _ in range(2):
        m._geo_grid_pts.grad = torch.randn_like(m._geo_grid_pts)
        m._sh0.grad = torch.randn_like(m._sh0)
        m.optimizer.step()
    m.optimizer_save_iteration(3)
    saved = m.optimizer.state_dict()
    m2 = _Model()
    m2.load(os.path.join(HERE, "ref_ckpt.pt"))
    m2.model_path = str(tmp_path)
    m2.optimizer = SparseAdam([{"params": [m2._geo_grid_pts], "lr": 0.01, "name": "_geo_grid_pts"},
                               {"params": [m2._sh0], "lr": 0.01, "name": "_sh0"}], betas=(0.1, 0.99))
    m2.optimizer_load_iteration(3)
    back = m2.optimizer.state_dict()
    for pid, st in saved["state"].items():
        assert back["state"][pid]["step"] == st["step"]
        assert torch.equal(back["state"][pid]["exp_avg"], st["exp_avg"])
        assert torch.equal(back["state"][pid]["exp_avg_sq"], st["exp_avg_sq"])
