"""Golden vectors for pruning / subdivision from the reference's own torch code.

Executes src/utils/octree_utils.py, src/utils/activation_utils.py and
src/sparse_voxel_gears/adaptive.py of the reference in place on the CPU (their "cuda" device
strings mapped to "cpu"; nothing is copied into this repository) on the seeded tiny scene, and
writes tests/golden/adaptive.npz: the grid-point link, gen_children + octpath_decoding,
subdivide_by_interp, agg_voxel_into_grid_pts, and a model subdivided then pruned by the
reference's SVAdaptive.

Usage (this machine, with the reference sources):
    python tests/golden/make_golden_adaptive.py [/path/to/reference]
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests.golden.adaptive_cases import model_inputs, scene, SUBDIV_FRAC, PRUNE_FRAC, OUTSIDE_LEVEL  # noqa: E402
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
    act = load_on_cpu(os.path.join(ref, "src", "utils", "activation_utils.py"), "src.utils.activation_utils")
    sys.modules["src.utils.activation_utils"] = act
    sys.modules["src.utils"].activation_utils = act
    octu = load_on_cpu(os.path.join(ref, "src", "utils", "octree_utils.py"), "src.utils.octree_utils")
    sys.modules["src.utils.octree_utils"] = octu
    sys.modules["src.utils"].octree_utils = octu
    adapt = load_on_cpu(os.path.join(ref, "src", "sparse_voxel_gears", "adaptive.py"), "ref_adaptive")

    sc = scene()
    out = {"digest": np.array(sc.n_vox)}
    octpath = torch.from_numpy(sc.octpath.reshape(-1, 1))
    octlevel = torch.from_numpy(sc.octlevel.reshape(-1, 1).astype(np.int8))
    key, vkey = octu.build_grid_pts_link(octpath, octlevel)
    out["link_key"], out["link_vox_key"] = key.numpy(), vkey.numpy()

    sel = torch.arange(0, sc.n_vox, 3)
    cp, cl = octu.gen_children(octpath[sel], octlevel[sel])
    cc, cs = octu.octpath_decoding(cp, cl, torch.zeros(3), torch.tensor([2.0]))
    out.update(child_path=cp.numpy(), child_level=cl.numpy(), child_center=cc.numpy(), child_size=cs.numpy())

    rng = np.random.default_rng(5)
    for c in (1, 3):
        v = torch.from_numpy(rng.normal(size=(200, 8, c)).astype(np.float32))
        out[f"interp_in_{c}"] = v.numpy()
        out[f"interp_out_{c}"] = adapt.subdivide_by_interp(v).numpy()
    aval = torch.from_numpy(rng.normal(size=(sc.n_vox, 8, 2)).astype(np.float32))
    out["agg_in"] = aval.numpy()
    out["agg_out"] = adapt.agg_voxel_into_grid_pts(len(key), vkey, aval).numpy()

    class Model(adapt.SVAdaptive):
        pass

    m = Model()
    inp = model_inputs(sc)
    for k, v in inp.items():
        setattr(m, k, torch.from_numpy(v) if isinstance(v, np.ndarray) else v)
    m.scene_center, m.scene_extent = torch.zeros(3), torch.tensor([2.0])
    m.outside_level = OUTSIDE_LEVEL
    m.per_voxel_attr_lst = ["octpath", "octlevel", "vox_center", "vox_size", "subdiv_meta", "is_leaf"]
    m.per_voxel_param_lst = ["_sh0", "_shs", "_subdiv_p"]
    m.grid_pts_param_lst = ["_geo_grid_pts"]
    m.grid_pts_key, m.vox_key = key, vkey
    sub = torch.from_numpy(np.random.default_rng(6).random(sc.n_vox) < SUBDIV_FRAC)
    m.subdividing(sub)
    names = m.per_voxel_attr_lst + m.per_voxel_param_lst + m.grid_pts_param_lst + ["vox_key", "grid_pts_key"]
    for n in names:
        out["sub_" + n] = getattr(m, n).detach().numpy()
    prune = torch.from_numpy(np.random.default_rng(7).random(len(m.octpath)) < PRUNE_FRAC)
    m.pruning(prune)
    for n in names:
        out["prune_" + n] = getattr(m, n).detach().numpy()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "adaptive.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, "voxels", sc.n_vox, "after subdivision", len(out["sub_octpath"]),
          "after pruning", len(out["prune_octpath"]), "kept parents", int((~out["sub_is_leaf"]).sum()))


if __name__ == "__main__":
    main()
