"""CPU checks of the native batched step's C surface (svr_step_*): the public header builds as
plain C11 with warnings as errors, the ctypes mirror of svr_step_desc_t has the C compiler's
layout, and bad arguments come back as SVR_ERR_ARG before any CUDA call."""
import ctypes as C

import pytest

from svraster_b200 import _lib
from tests import native_host


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    return native_host.compile_driver(str(tmp_path_factory.mktemp("native_host")))


def test_descriptor_layout_matches_c(driver):
    lay = native_host.layout(driver)
    assert lay.pop("sizeof") == C.sizeof(_lib.StepDesc)
    assert lay.pop("view_sizeof") == C.sizeof(_lib.ViewDesc)
    assert lay == {name: getattr(_lib.StepDesc, name).offset for name, _ in _lib.StepDesc._fields_}


def _desc(**over):
    d = _lib.StepDesc()
    d.n_vox, d.sh_degree, d.grid_res_pow2, d.n_grid = 8, 3, 4, 27
    for name in ("octpath", "centers", "lengths", "is_leaf", "vox_key", "grid", "sh0", "shs", "s_val"):
        setattr(d, name, 0x1000)          # never dereferenced: the checks below fail first
    d.inside_extent = 2.0
    for k, v in over.items():
        setattr(d, k, v)
    return d


def _views(n=1):
    arr = (_lib.ViewDesc * n)()
    for v in arr:
        v.width, v.height, v.w2c, v.c2w = 16, 16, 0x1000, 0x1000
    return arr


@pytest.mark.parametrize("over", [dict(n_vox=0), dict(sh_degree=4), dict(grid_res_pow2=0), dict(grid_res_pow2=11),
                                  dict(inside_extent=0.0), dict(n_grid=0), dict(octpath=None), dict(grid=None),
                                  dict(adam_rows=-1), dict(record_capacity=-5)])
def test_create_rejects_bad_descriptors(over):
    L = _lib.load()
    h = C.c_void_p(7)
    assert L.svr_step_create(C.byref(_desc(**over)), _views(), 1, None, C.byref(h)) == -1
    assert h.value is None                 # the handle is cleared on failure


def test_create_rejects_bad_views():
    L = _lib.load()
    h = C.c_void_p()
    assert L.svr_step_create(C.byref(_desc()), _views(), 0, None, C.byref(h)) == -1
    assert L.svr_step_create(C.byref(_desc()), _views(), 129, None, C.byref(h)) == -1
    bad = _views()
    bad[0].c2w = None
    assert L.svr_step_create(C.byref(_desc()), bad, 1, None, C.byref(h)) == -1
    assert L.svr_step_create(None, _views(), 1, None, C.byref(h)) == -1
    assert L.svr_step_create(C.byref(_desc()), _views(), 1, None, None) == -1


def test_null_handles():
    L = _lib.load()
    p, n = C.c_void_p(), C.c_int64()
    r, o = C.c_uint32(), C.c_uint32()
    assert L.svr_step_run(None, 3, None) == -1
    assert L.svr_step_capture(None, None) == -1
    assert L.svr_step_buffer(None, 0, C.byref(p), C.byref(n)) == -1
    assert L.svr_step_info(None, (C.c_int64 * 8)()) == -1
    assert L.svr_step_status(None, C.byref(r), C.byref(o), None) == -1
    assert L.svr_step_destroy(None) == 0


def test_python_buffer_names_match_the_header_enum():
    import os
    import re
    from svraster_b200 import native_step
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "svraster_b200.h")).read()
    enum = {m.group(1).lower(): int(m.group(2)) for m in re.finditer(r"SVR_STEP_([A-Z0-9_]+) = (\d+)", hdr)}
    n = enum.pop("n_buffers")
    assert len(native_step.BUFFERS) == n == len(enum)
    assert {k.lower(): v for k, v in native_step.BUFFERS.items()} == enum
    assert (native_step.GRADS, native_step.ADAM) == (1, 2)


def test_binning_buffer_holds_a_candidate_row_block_per_tile_and_per_slot():
    """svr_binning_buffer_bytes(R, T) includes the candidate rows: 4 KB per slot of 128
    records plus 4 KB per tile (a tile's partial slot)."""
    lib = _lib.load()
    R = 1_000_000
    assert lib.svr_binning_buffer_bytes(R, 101) - lib.svr_binning_buffer_bytes(R, 100) == 4096
    assert lib.svr_binning_buffer_bytes(R + 128 * 10, 100) - lib.svr_binning_buffer_bytes(R, 100) >= 10 * 4096
