"""The C-ABI library loads without a GPU, exports every symbol ``include/glide_b200.h``
declares, agrees with the ctypes struct layouts, and rejects invalid arguments
with a status and an error text before touching the device."""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

from glide_b200 import _abi

HEADER = Path(__file__).resolve().parents[1] / "include" / "glide_b200.h"


def declared_functions() -> set[str]:
    text = HEADER.read_text()
    return set(re.findall(r"^\s*(?:glide_status|int32_t)\s+(glide_\w+)\s*\(", text, re.M))


def test_header_declares_what_the_binding_binds():
    assert declared_functions() == set(_abi.SIGNATURES)


def test_every_symbol_is_exported():
    lib = C.CDLL(str(_abi.LIB_PATH))
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_struct_layouts_match():
    sizes = (C.c_size_t * len(_abi.STRUCTS))()
    assert _abi.lib.glide_abi_struct_sizes(sizes, len(_abi.STRUCTS)) == 0
    assert list(sizes) == [C.sizeof(s) for s in _abi.STRUCTS]
    assert _abi.lib.glide_version() >= 100


def test_invalid_arguments_are_rejected_without_a_device():
    assert _abi.lib.glide_step(None, None) == 1
    assert "NULL" in _abi.last_error()
    a = _abi.StepArgs()
    a.n = 10
    a.n_steps = 1
    assert _abi.lib.glide_step(C.byref(a), None) == 1
    assert "NULL" in _abi.last_error()
    a.n_steps = 0
    assert _abi.lib.glide_step(C.byref(a), None) == 1
    assert "n_steps" in _abi.last_error()
    w = _abi.WindowDesc()
    assert _abi.lib.glide_window_pack(C.byref(w), None) == 1
    c = _abi.ConvectArgs()
    assert _abi.lib.glide_convect(C.byref(c), None) == 1
    nb = C.c_size_t()
    assert _abi.lib.glide_convect_scratch_bytes(1, C.byref(nb)) == 1
    assert _abi.lib.glide_convect_scratch_bytes(60, C.byref(nb)) == 0
    assert nb.value == 8 * (8 + 4 * 60 + 60 * 60)
    wb, sb, pb = C.c_size_t(), C.c_size_t(), C.c_size_t()
    assert _abi.lib.glide_window_packed_bytes(60, 281, 401, 0, C.byref(wb), C.byref(sb), C.byref(pb)) == 0
    assert wb.value == 60 * 281 * 401 * 32 and sb.value == 281 * 401 * 64
    assert _abi.lib.glide_window_packed_bytes(60, 281, 401, 7, C.byref(wb), C.byref(sb), C.byref(pb)) == 3
    r = _abi.RegridArgs()
    assert _abi.lib.glide_agl_regrid(C.byref(r), None) == 1 and "sizes" in _abi.last_error()
    levels = (C.c_double * 3)(0.0, 50.0, 20.0)  # not ascending
    r.n_channels, r.zp, r.za, r.ny, r.nx = 1, 4, 3, 2, 2
    r.height_agl_p = r.fields_p = r.fields_agl = r.scratch = 64
    r.agl_levels = C.cast(levels, C.c_void_p)
    assert _abi.lib.glide_agl_regrid(C.byref(r), None) == 1 and "ascending" in _abi.last_error()
    assert _abi.lib.glide_agl_regrid_scratch_bytes(3, 2, 2, C.byref(nb)) == 0 and nb.value == 3 * 4 * 12 + 32


def test_check_raises_with_text():
    with pytest.raises(_abi.GlideError, match="args is NULL"):
        _abi.check(_abi.lib.glide_step(None, None), "glide_step")


def test_empty_launch_is_a_no_op_without_a_device():
    a = _abi.StepArgs()
    a.n = 0
    a.n_steps = 1
    assert _abi.lib.glide_step(C.byref(a), None) == 0
    c = _abi.ConvectArgs()
    c.n, c.nz, c.ny, c.nx = 0, 4, 2, 2
    assert _abi.lib.glide_convect(C.byref(c), None) == 1  # met inputs are still required


def test_footprint_compact_arguments_are_checked_without_a_device():
    nb = C.c_size_t()
    lib = _abi.lib
    assert lib.glide_footprint_compact_scratch_bytes(3, 4097, C.byref(nb)) == 0
    assert nb.value == 8 * (3 * 3 + 1) + 4 * 3 * 3  # 3 tiles of 2048 cells per slice
    assert lib.glide_footprint_compact_scratch_bytes(0, 1, C.byref(nb)) == 0 and nb.value == 8
    assert lib.glide_footprint_compact_scratch_bytes(-1, 10, C.byref(nb)) == 1 and "negative" in _abi.last_error()
    assert lib.glide_footprint_compact_scratch_bytes(1, 0, C.byref(nb)) == 1 and "cells" in _abi.last_error()
    assert lib.glide_footprint_compact_scratch_bytes(1, 2**31, C.byref(nb)) == 1
    assert lib.glide_footprint_compact_scratch_bytes(2**30, 2**20, C.byref(nb)) == 1 and "tiles" in _abi.last_error()
    assert lib.glide_footprint_compact(None, None) == 1 and "NULL" in _abi.last_error()
    a = _abi.CompactArgs()
    a.k, a.cells, a.n_rows, a.capacity = 2, 100, 4, 200
    assert lib.glide_footprint_compact(C.byref(a), None) == 1 and "NULL" in _abi.last_error()
    a.rows = a.row_index = a.slice_offset = a.out_cell = a.out_value = 64
    a.scratch, a.scratch_bytes = 64, 8
    assert lib.glide_footprint_compact(C.byref(a), None) == 1 and "scratch" in _abi.last_error()
    a.scratch_bytes = 1024
    a.row_index = 68  # not 8-byte aligned
    assert lib.glide_footprint_compact(C.byref(a), None) == 1 and "misaligned" in _abi.last_error()
    a.row_index = 64
    a.capacity = -1
    assert lib.glide_footprint_compact(C.byref(a), None) == 1 and "capacity" in _abi.last_error()
    a.capacity, a.n_rows = 200, 2**62
    assert lib.glide_footprint_compact(C.byref(a), None) == 1 and "n_rows" in _abi.last_error()
    a.n_rows, a.capacity, a.out_cell = 4, 10, None
    assert lib.glide_footprint_compact(C.byref(a), None) == 1 and "capacity > 0" in _abi.last_error()
