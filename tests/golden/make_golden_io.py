"""Golden vectors for the checkpoint formats from the reference's own code.

Executes src/sparse_voxel_gears/io.py of the reference in place on the CPU ("cuda" device
strings mapped to "cpu"; nothing is copied into this repository) and writes:

* tests/golden/io_quant.npz -- quantization() (the 8-bit codebook of a saved checkpoint,
  io.py:123-167) on the seeded value sets of ``io_cases.QUANT_CASES``: index and codebook;
* tests/golden/ref_ckpt.pt, tests/golden/ref_ckpt_q.pt -- SVInOut.save (io.py:18-48) of the
  seeded small model of ``io_cases.model_fields``, plain and quantized.

Usage (this machine, with the reference sources):
    python tests/golden/make_golden_io.py [/path/to/reference]
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests.golden.io_cases import QUANT_CASES, model_fields, quant_values  # noqa: E402
from tests.golden.make_golden_extract import load_on_cpu  # noqa: E402


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SVR_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: give the reference checkout as the first argument or in SVR_REFERENCE_DIR")
    import svraster_b200
    svraster_b200.install_as_svraster_cuda()
    for name in ("src", "src.utils"):
        m = types.ModuleType(name)
        m.__path__ = []
        sys.modules[name] = m
    sys.modules["src.utils.octree_utils"] = types.ModuleType("src.utils.octree_utils")
    sys.modules["src.utils"].octree_utils = sys.modules["src.utils.octree_utils"]
    io = load_on_cpu(os.path.join(ref, "src", "sparse_voxel_gears", "io.py"), "ref_io")
    here = os.path.dirname(os.path.abspath(__file__))

    out = {}
    for name in QUANT_CASES:
        v = torch.from_numpy(quant_values(name))
        q = io.quantization(v)
        out[f"{name}_index"] = q["index"].numpy()
        out[f"{name}_codebook"] = q["codebook"].numpy()
    np.savez_compressed(os.path.join(here, "io_quant.npz"), **out)

    class Model(io.SVInOut):
        pass

    for quant, fname in ((False, "ref_ckpt.pt"), (True, "ref_ckpt_q.pt")):
        m = Model()
        for k, v in model_fields().items():
            setattr(m, k, torch.from_numpy(v) if isinstance(v, np.ndarray) else v)
        m.save(os.path.join(here, fname), quantize=quant)
    print("wrote", sorted(out), "and 2 checkpoints")


if __name__ == "__main__":
    main()
