"""CPU-side checks of the C-ABI library: it loads and exports every declared entry point."""
import os
import re

import pytest

from svraster_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "svraster_b200.h")).read()
    return sorted(set(re.findall(r"SVR_API\s+[\w\s\*]+?\b(svr_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ["svr_preprocess", "svr_bin_and_sort", "svr_render_fwd", "svr_render_bwd", "svr_gather_geo",
              "svr_sh_eval", "svr_laplacian_bw", "svr_eikonal_bw", "svr_adam_step", "svr_valid_table_fill"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), f"{name} not exported"
    assert set(_lib.exported_symbols()) >= set(declared_symbols())


def test_buffer_size_queries_are_monotone():
    lib = _lib.load()
    assert lib.svr_geom_buffer_bytes(10_000) >= lib.svr_geom_buffer_bytes(100)
    assert lib.svr_binning_buffer_bytes(1_000_000, 100) >= 80 * 1_000_000
    assert lib.svr_image_buffer_bytes(640 * 480, 1200) >= 4 * 640 * 480 + 12 * 1200
    assert lib.svr_version() >= 1


def test_view_descriptor_layout():
    import ctypes as C
    assert C.sizeof(_lib.ViewDesc) == 80


def test_null_arguments_are_rejected_before_any_cuda_call():
    """Null pointers come back as SVR_ERR_ARG (-1) from the argument checks, before the entry
    point reaches the CUDA runtime (without a GPU any runtime call would fail with -2)."""
    lib = _lib.load()
    # svr_grid_index_build(G, grid_keys, grid_res, dense_index, status, stream)
    assert lib.svr_grid_index_build(10, None, 64, None, None, None) == -1
    # svr_laplacian_bw_noalloc(G, A, active, grid_keys, grid2voxel, grid_res, grid_mask, voxel_coords,
    #     voxel_sizes, N, vox_key, grid_pts, M, weight, vox_size_inv, seed, grid_grad, status, stream)
    # with A > 0 and every pointer null
    args = [10, 5, None, None, None, 64, None, None, None, 0, None, None, 0, 0.01, 1.0, 1, None, None, None]
    assert len(args) == 19
    assert lib.svr_laplacian_bw_noalloc(*args) == -1
    args[5] = 0                        # grid_res <= 0: a bad argument
    assert lib.svr_laplacian_bw_noalloc(*args) == -1
    args[5] = 256                      # above the static index: capacity
    assert lib.svr_laplacian_bw_noalloc(*args) == -3


def test_candidate_row_query_rejects_null_arguments():
    import ctypes as C
    lib = _lib.load()
    v = C.c_int(7)
    assert lib.svr_binning_candidates_valid(None, C.byref(v), None) == -1
    assert v.value == 7


def test_binding_argument_counts_match_the_header():
    """Every ctypes signature in _lib has as many arguments as the header's prototype."""
    src = open(os.path.join(ROOT, "include", "svraster_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    protos = {}
    for m in re.finditer(r"SVR_API\s+[\w\s\*]+?\b(svr_\w+)\s*\(([^;]*?)\)\s*;", src, flags=re.S):
        params = m.group(2).strip()
        protos[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    assert set(protos) == set(declared_symbols())
    for name, n in protos.items():
        assert name in _lib._SIGS, f"{name} has no ctypes signature"
        assert len(_lib._SIGS[name][1]) == n, f"{name}: header has {n} arguments, binding {len(_lib._SIGS[name][1])}"


def test_binding_argument_types_match_the_header():
    """Scalar arguments have the header's width (int / int64_t / size_t / float / double /
    uint64_t), pointers are bound as pointers."""
    import ctypes as C
    src = open(os.path.join(ROOT, "include", "svraster_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    scalar = {"int": C.c_int, "int32_t": C.c_int, "int64_t": C.c_int64, "uint64_t": C.c_uint64,
              "size_t": C.c_size_t, "float": C.c_float, "double": C.c_double, "uint32_t": C.c_uint32}
    for m in re.finditer(r"SVR_API\s+[\w\s\*]+?\b(svr_\w+)\s*\(([^;]*?)\)\s*;", src, flags=re.S):
        name, params = m.group(1), m.group(2).strip()
        if params in ("", "void"):
            continue
        bound = _lib._SIGS[name][1]
        for i, (param, ct) in enumerate(zip(params.split(","), bound)):
            p = " ".join(param.replace("const", " ").split())
            if "*" in p:
                assert ct in (C.c_void_p, C.c_char_p) or hasattr(ct, "_type_") and ct.__name__.startswith("LP_"), \
                    f"{name} argument {i} ({param.strip()}) is a pointer, bound as {ct}"
            else:
                base = p.split()[0]
                assert base in scalar, f"{name} argument {i}: unknown type {param.strip()}"
                assert C.sizeof(ct) == C.sizeof(scalar[base]) and \
                    (ct in (C.c_float, C.c_double)) == (scalar[base] in (C.c_float, C.c_double)), \
                    f"{name} argument {i} ({param.strip()}) bound as {ct}"
