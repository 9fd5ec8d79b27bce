"""B200 (sm_100a) implementation of SVRecon's sparse-voxel SDF rasterizer path.

The package mirrors the ``svraster_cuda`` Python surface (cuda/svraster_cuda/__init__.py:1-6):
``meta``, ``utils``, ``renderer``, ``sparse_adam``, ``marching_cubes`` and ``grid_loss_bw``.
``install_as_svraster_cuda()`` registers it under that name so existing callers
(train.py, extract_mesh_sdf.py) import it unchanged.
"""
import sys

from . import meta
from . import renderer
from . import utils
from . import sparse_adam
from . import grid_loss_bw
from . import marching_cubes

__all__ = ["meta", "renderer", "utils", "sparse_adam", "grid_loss_bw", "marching_cubes",
           "install_as_svraster_cuda"]


def install_as_svraster_cuda():
    """Make ``import svraster_cuda`` (and its submodules) resolve to this package."""
    pkg = sys.modules[__name__]
    sys.modules["svraster_cuda"] = pkg
    for name in ("meta", "utils", "renderer", "sparse_adam", "grid_loss_bw", "marching_cubes"):
        sys.modules[f"svraster_cuda.{name}"] = getattr(pkg, name)
    return pkg
