"""Drop-in replacement of ``svraster_cuda.marching_cubes`` (cuda/svraster_cuda/marching_cubes.py)."""
from __future__ import annotations


def torch_marching_cubes_grid(grid_pts_val, grid_pts_xyz, vox_key, iso, chunk_sz=10_000_000):
    raise NotImplementedError("sparse marching cubes kernel not built yet")
