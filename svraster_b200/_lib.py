"""ctypes binding of ``libsvraster_b200.so`` (the C ABI in ``include/svraster_b200.h``).

Torch is used only for device memory and the current CUDA stream: every call passes raw
device pointers and ``torch.cuda.current_stream().cuda_stream``.  There is no fallback:
if the library is missing or cannot load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsvraster_b200.so")

SVR_MAX_VIEWS = 128
TILE = 16


class ViewDesc(C.Structure):
    """Mirror of ``svr_view_t``."""
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32),
        ("tiles_x", C.c_int32), ("tiles_y", C.c_int32),
        ("tile_offset", C.c_int32), ("pad0", C.c_int32),
        ("pix_offset", C.c_int64),
        ("tanfovx", C.c_float), ("tanfovy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
        ("near_plane", C.c_float), ("pad1", C.c_float),
        ("w2c", C.c_void_p), ("c2w", C.c_void_p), ("bg", C.c_void_p),
    ]


class StepDesc(C.Structure):
    """Mirror of ``svr_step_desc_t`` (natural alignment, as the C compiler lays it out)."""
    _fields_ = [
        ("n_vox", C.c_int32), ("sh_degree", C.c_int32), ("sh_bf16", C.c_int32), ("grid_res_pow2", C.c_int32),
        ("octpath", C.c_void_p), ("centers", C.c_void_p), ("lengths", C.c_void_p), ("is_leaf", C.c_void_p),
        ("vox_key", C.c_void_p), ("grid", C.c_void_p), ("sh0", C.c_void_p), ("shs", C.c_void_p),
        ("n_grid", C.c_int64), ("s_val", C.c_void_p),
        ("scene_center", C.c_float * 3), ("inside_extent", C.c_float),
        ("lambda_ls", C.c_float), ("lambda_ge", C.c_float), ("lambda_R_concen", C.c_float),
        ("lr", C.c_double * 3), ("beta1", C.c_double), ("beta2", C.c_double), ("eps", C.c_float),
        ("seed", C.c_int32), ("adam_rows", C.c_int32), ("record_capacity", C.c_int64),
    ]


_P, _I, _I64, _U64, _F, _D, _SZ = C.c_void_p, C.c_int, C.c_int64, C.c_uint64, C.c_float, C.c_double, C.c_size_t

_SIGS = {
    "svr_last_error": (C.c_char_p, []),
    "svr_version": (_I, []),
    "svr_kernel_launches": (C.c_longlong, []),
    "svr_scatter_vox_grads": (_I, [_I64, _I, _P, _P, _P, _P]),
    "svr_sh_eval_views": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "svr_sh_eval_views_bw": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "svr_sh_eval_views_bw_add": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "svr_geom_buffer_bytes": (_SZ, [_I64]),
    "svr_preprocess": (_I, [_P, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "svr_unpack_geom": (_I, [_P, _I64, _P, _P, _P, _P]),
    "svr_count_rendered": (_I, [_I64, _P, C.POINTER(C.c_int64), C.POINTER(C.c_uint64), _P]),
    "svr_scan_rendered": (_I, [_I64, _P, _P]),
    "svr_render_fwd_max_w_views": (_I, [_P, _I, _I, _I64, _I, _I, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P,
                                        _P, _P, _P]),
    "svr_grid_link_workspace_bytes": (C.c_size_t, [_I64]),
    "svr_grid_link": (_I, [_I64, _P, _P, _P, C.c_size_t, _P, _P, C.POINTER(C.c_int64), _P, _P]),
    "svr_subdivide_interp": (_I, [_I64, _I, _P, _P, _P]),
    "svr_agg_voxel_into_grid_pts": (_I, [_I64, _I, _P, _P, _I64, _P, _P, _P, _P]),
    "svr_training_stat_reduce": (_I, [_I, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "svr_render_config_count": (_I, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "svr_render_config_describe": (_I, [_I, _I, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "svr_render_set_config": (_I, [_I, _I]),
    "svr_render_get_config": (_I, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "svr_binning_count": (_I, [_P, C.POINTER(C.c_int64), _P]),
    "svr_binning_candidates_valid": (_I, [_P, C.POINTER(C.c_int), _P]),
    "svr_workspace_query": (_I, [_I, _I, _I64, _I64, _I, C.POINTER(C.c_size_t)]),
    "svr_binning_buffer_bytes": (_SZ, [_I64, _I]),
    "svr_image_buffer_bytes": (_SZ, [_I64, _I]),
    "svr_bin_and_sort": (_I, [_P, _I, _I, _I64, _U64, _P, _P, _P, _SZ, _P, _P]),
    "svr_bin_and_sort_ranked": (_I, [_P, _I, _I, _I64, _U64, _P, _P, _I, _P, _P, _SZ, _P, _P]),
    "svr_rank_table_workspace_bytes": (_I, [_I64, C.POINTER(C.c_size_t)]),
    "svr_rank_table_build": (_I, [_I64, _P, _U64, _P, C.POINTER(C.c_int), _P, _SZ, _P]),
    "svr_unpack_binning": (_I, [_P, _I64, _I, _P, _I64, _P, _P, _P, _P, _P]),
    "svr_render_set_impl": (_I, [_I, _I]),
    "svr_render_get_impl": (_I, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "svr_set_pack_event": (_I, [_P]),
    "svr_rendered_total": (_I, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_uint64), _P]),
    "svr_bin_tiles": (_I, [_P, _I, _I, _I64, _P, _I, _P, _P, _SZ, _P, _P]),
    "svr_pair_order_build": (_I, [_I64, _P, _P, C.POINTER(C.c_int), _P, _SZ, _P]),
    "svr_render_fwd_count_pairs": (_I, [_P, _I, _I, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "svr_render_fwd": (_I, [_P, _I, _I, _I64, _I, _I, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P,
                            _P, _P, _P, _P, _P, _P]),
    "svr_render_bwd": (_I, [_P, _I, _I, _I64, _I, _I, _F, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                            _P, _P, _P, _P]),
    "svr_read_status": (_I, [_P, _I64, _I, C.POINTER(C.c_uint32), _P]),
    "svr_gather_geo": (_I, [_I64, _P, _P, _P, _P, _P]),
    "svr_gather_geo_bw": (_I, [_I64, _P, _P, _P, _P, _P]),
    "svr_sh_eval": (_I, [_I, _I64, _P, _I, _I, _P, _P, _P, _P, _P, _P]),
    "svr_sh_eval_bw": (_I, [_I, _I64, _P, _I, _I, _P, _P, _P, _P, _P, _P]),
    "svr_valid_table_workspace_bytes": (_SZ, [_I, _I64]),
    "svr_valid_table_count": (_I, [_I, _P, _P, _P, _F, _I, _P, _P, C.POINTER(C.c_int64), _P]),
    "svr_valid_table_fill": (_I, [_I, _P, _P, _P, _F, _I, _P, _I64, _P, _P, _P, _P, _P]),
    "svr_grid_index_build": (_I, [_I, _P, _I, _P, _P, _P]),
    "svr_laplacian_bw": (_I, [_I, _I, _P, _P, _P, _I, _P, _P, _P, _P, _I, _P, _P, _I, _F, _F, _I, _P, _P, _P]),
    "svr_laplacian_bw_at_step": (_I, [_I, _I, _P, _P, _P, _I, _P, _P, _P, _P, _I, _P, _P, _I, _F, _F, _I, _P, _P, _P,
                                      _P]),
    "svr_voxel_gradient_bw": (_I, [_I, _I, _P, _P, _P, _I64, _P, _F, _P, _P, _P]),
    "svr_total_variation_bw": (_I, [_I64, _I, _P, _P, _I64, _F, _P, _I, _I, _P, _P, _P, _P]),
    "svr_points_loss_bw": (_I, [_I, _P, _I, _P, _P, _I, _P, _P, _P, _P, _I, _P, _P, _I, _F, _P, _P, _P]),
    "svr_normal_depth_loss": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P, _P]),
    "svr_quantize_workspace_bytes": (_I, [_I64, C.POINTER(C.c_size_t)]),
    "svr_quantize": (_I, [_I64, _P, _I, _P, _P, _P, _SZ, C.POINTER(C.c_int), _P, _P]),
    "svr_dequantize": (_I, [_I64, _P, _P, _P, _P]),
    "svr_voxel_order_workspace_bytes": (_I, [_I64, C.POINTER(C.c_size_t)]),
    "svr_voxel_order": (_I, [_I64, _P, _I64, _P, _P, _P, _SZ, _P, _P]),
    "svr_voxel_gradient_bw_ordered": (_I, [_I, _I, _P, _P, _P, _P, _P, _I64, _P, _F, _P, _P, _P, _P]),
    "svr_total_variation_bw_ordered": (_I, [_I64, _I, _P, _P, _P, _I64, _F, _P, _I, _I, _P, _P, _P, _P]),
    "svr_smoothness_bw_vox": (_I, [_I, _I, _P, _P, _P, _I, _P, _P, _P, _P, _I, _P, _F, _F, _F, _I, _P, _P, _I, _P,
                                   _P]),
    "svr_eikonal_bw_at_step": (_I, [_I, _I, _P, _P, _P, _I, _P, _P, _P, _P, _I, _P, _P, _I, _F, _F, _I, _P, _P, _P,
                                    _P]),
    "svr_eikonal_bw": (_I, [_I, _I, _P, _P, _P, _I, _P, _P, _P, _P, _I, _P, _P, _I, _F, _F, _I, _P, _P, _P]),
    "svr_laplacian_bw_noalloc": (_I, [_I, _I, _P, _P, _P, _I, _P, _P, _P, _I, _P, _P, _I, _F, _F, _I, _P, _P, _P]),
    "svr_tsdf_integrate": (_I, [_P, _P, _I, _I64, _P, _P, _I, _I, _P, _I, _I, _I, _P, _D, _D, _F, _I, _I, _I, _F,
                                _I, _P, _P, _P]),
    "svr_mc_workspace_bytes": (_SZ, [_I64, _I64]),
    "svr_mc_count": (_I, [_I64, _P, _I64, _P, _F, _P, C.POINTER(C.c_int64), _P]),
    "svr_mc_emit": (_I, [_I64, _P, _P, _P, _F, _I64, _I, _P, _P, _P, C.POINTER(C.c_int64), _P]),
    "svr_adam_step": (_I, [_I64, _I, _I, _P, _P, _P, _P, _D, _D, _D, _D, _F, _P]),
    "svr_adam_coef_table": (_I, [_I, _D, _D, _D, _I64, _P]),
    "svr_sh_eval_views_bf16": (_I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "svr_adam_step_bf16": (_I, [_I64, _I, _I, _P, _P, _P, _P, _D, _D, _D, _D, _F, _P]),
    "svr_adam_step_bf16_at": (_I, [_I64, _I, _I, _P, _P, _P, _P, _P, _I64, _P, _D, _D, _F, _P, _P]),
    "svr_adam_step_at": (_I, [_I64, _I, _I, _P, _P, _P, _P, _P, _I64, _P, _D, _D, _F, _P, _P]),
    "svr_counter_add": (_I, [_P, _I64, _P]),
    "svr_step_create": (_I, [_P, _P, _I, _P, C.POINTER(C.c_void_p)]),
    "svr_step_destroy": (_I, [_P]),
    "svr_step_buffer": (_I, [_P, _I, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]),
    "svr_step_info": (_I, [_P, _P]),
    "svr_step_run": (_I, [_P, _I, _P]),
    "svr_step_capture": (_I, [_P, _P]),
    "svr_step_status": (_I, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), _P]),
}

_lib = None


def load():
    """Load the CUDA library once; raise if it is missing (there is no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"svraster_b200: CUDA library not built ({LIB_PATH}); run svraster_b200/build.py")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    return list(_SIGS)


class SvrError(RuntimeError):
    pass


def check(rc: int, what: str):
    if rc != 0:
        msg = load().svr_last_error().decode(errors="replace")
        raise SvrError(f"{what} failed (status {rc}): {msg}")


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_ptr(device=None):
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(*tensors):
    for t in tensors:
        if t is not None and torch.is_tensor(t) and not t.is_cuda:
            raise SvrError("svraster_b200 operates on CUDA tensors only")


def make_views(cams):
    """Build a ctypes array of ViewDesc from dicts with keys width, height, tanfovx, tanfovy,
    cx, cy, near, w2c, c2w, bg (the last three device float32 tensors)."""
    n = len(cams)
    if n == 0 or n > SVR_MAX_VIEWS:
        raise SvrError(f"view count must be in 1..{SVR_MAX_VIEWS}")
    arr = (ViewDesc * n)()
    tile_off, pix_off = 0, 0
    for i, c in enumerate(cams):
        v = arr[i]
        v.width, v.height = int(c["width"]), int(c["height"])
        v.tiles_x, v.tiles_y = (v.width + TILE - 1) // TILE, (v.height + TILE - 1) // TILE
        v.tile_offset, v.pix_offset = tile_off, pix_off
        v.tanfovx, v.tanfovy = float(c["tanfovx"]), float(c["tanfovy"])
        v.cx, v.cy = float(c["cx"]), float(c["cy"])
        v.near_plane = float(c.get("near", 0.02))
        v.w2c, v.c2w, v.bg = ptr(c["w2c"]), ptr(c["c2w"]), ptr(c["bg"])
        tile_off += v.tiles_x * v.tiles_y
        pix_off += v.width * v.height
    return arr, tile_off, pix_off
