"""Checkpoint formats on the CPU: the oracle's 8-bit codebook against the reference's own
quantization() (tests/golden/io_quant.npz), the structure of checkpoints written by the
reference's SVInOut.save (tests/golden/ref_ckpt.pt, ref_ckpt_q.pt; both made by
tests/golden/make_golden_io.py), and the config.yaml dump."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from tests.golden.io_cases import QUANT_CASES, model_fields, quant_values

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return torch.load(os.path.join(HERE, name), map_location="cpu", weights_only=True)


@pytest.mark.parametrize("name", QUANT_CASES)
def test_oracle_codebook_matches_reference_bitexact(name):
    from oracle import oracle as O
    g = np.load(os.path.join(HERE, "io_quant.npz"))
    idx, book, _ = O.quantize(quant_values(name))
    assert idx.shape == g[f"{name}_index"].shape
    assert np.array_equal(idx, g[f"{name}_index"])
    assert np.array_equal(book.view(np.uint32), g[f"{name}_codebook"].view(np.uint32))


def test_reference_plain_checkpoint_holds_the_model():
    sd = _load("ref_ckpt.pt")
    f = model_fields()
    assert sd["quantized"] is False
    assert set(sd) == set(f) | {"quantized"}
    for k, v in f.items():
        if isinstance(v, np.ndarray):
            assert sd[k].numpy().dtype == v.dtype and np.array_equal(sd[k].numpy(), v), k
        else:
            assert sd[k] == v, k


def test_reference_quantized_checkpoint_layout_and_oracle_codebooks():
    """The quantized file: grid as one {index, codebook}, sh0 / shs as one per column of dim 1,
    each equal bit for bit to the oracle's codebook of that column."""
    from oracle import oracle as O
    sd = _load("ref_ckpt_q.pt")
    f = model_fields()
    assert sd["quantized"] is True
    assert isinstance(sd["_geo_grid_pts"], dict)
    assert isinstance(sd["_sh0"], list) and len(sd["_sh0"]) == f["_sh0"].shape[1]
    assert isinstance(sd["_shs"], list) and len(sd["_shs"]) == f["_shs"].shape[1]
    pieces = [(sd["_geo_grid_pts"], f["_geo_grid_pts"])]
    pieces += [(q, f["_sh0"][:, j:j + 1]) for j, q in enumerate(sd["_sh0"])]
    pieces += [(q, f["_shs"][:, j:j + 1]) for j, q in enumerate(sd["_shs"])]
    for q, vals in pieces:
        assert q["index"].dtype == torch.uint8 and tuple(q["index"].shape) == vals.shape
        assert q["codebook"].dtype == torch.float32 and q["codebook"].numel() == 256
        idx, book, _ = O.quantize(vals)
        assert np.array_equal(q["index"].numpy(), idx)
        assert np.array_equal(q["codebook"].numpy().view(np.uint32), book.view(np.uint32))


def test_config_dump_roundtrip(tmp_path):
    import yaml
    from svraster_b200 import io
    cfg = {"model": {"n_samp_per_vox": 3, "white_background": False, "model_path": "out/x"},
           "optimizer": {"geo_lr": 0.025, "lr_decay_ckpt": [19000, 23000], "optim_betas": (0.1, 0.99)},
           "regularizer": {"lambda_tv_density": 1e-8, "tv_sparse": False}}
    text = io.dump_config(cfg, str(tmp_path / "config.yaml"))
    assert text == yaml.safe_dump(io._plain(cfg))
    back = io.load_config(str(tmp_path / "config.yaml"))
    assert back["optimizer"]["optim_betas"] == [0.1, 0.99]
    assert back["model"] == cfg["model"] and back["regularizer"] == cfg["regularizer"]


def test_io_needs_cuda_without_a_gpu():
    from svraster_b200 import io
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA"):
        io.quantization(torch.zeros(4))
