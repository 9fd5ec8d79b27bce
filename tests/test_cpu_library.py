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
