"""The C ABI library loads, exports what include/hexdyn.h declares, and
refuses invalid descriptors before touching the device."""

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import hexdyn._lib as L

HEADER = Path(__file__).resolve().parent.parent / "include" / "hexdyn.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(hexdyn_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = L.load()
    names = declared()
    assert "hexdyn_step" in names and "hexdyn_create" in names
    for name in names:
        assert hasattr(lib, name), name
        assert name in L.EXPORTS, f"{name} missing from the ctypes binding"
    assert lib.hexdyn_abi_version() == L.HEXDYN_ABI_VERSION


def test_create_refuses_null_and_bad_sizes():
    lib = L.load()
    h = C.c_void_p()
    assert lib.hexdyn_create(None, C.byref(h)) == L.HEXDYN_E_ARG
    d = L.HexDynDesc()
    assert lib.hexdyn_create(C.byref(d), C.byref(h)) == L.HEXDYN_E_ARG
    assert "positive" in L.last_error()
    d.n_cells, d.n_edges, d.n_vertices, d.n_levels = 10, 30, 20, 2
    assert lib.hexdyn_create(C.byref(d), C.byref(h)) == L.HEXDYN_E_ARG
    assert "n_levels" in L.last_error()


def test_calls_on_null_handle_are_refused():
    lib = L.load()
    x = np.zeros(4, dtype=np.float32)
    assert lib.hexdyn_set_state(None, 0, x.ctypes.data_as(C.POINTER(C.c_float)), 4, None) == L.HEXDYN_E_ARG
    assert lib.hexdyn_step(None, None, 1, None, None) == L.HEXDYN_E_ARG
    ptrs = (C.c_void_p * L.HEXDYN_NUM_FIELDS)()
    assert lib.hexdyn_step_host(None, ptrs, ptrs, None) == L.HEXDYN_E_ARG
    assert lib.hexdyn_destroy(None) == L.HEXDYN_OK


def test_struct_matches_header_field_order():
    text = HEADER.read_text()
    body = text[text.index("typedef struct HexDynDesc"):text.index("} HexDynDesc;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = re.findall(r"\b([a-z_0-9]+)(?:\[3\])?\s*[,;]", body)
    assert [n for n in names] == [f[0] for f in L.HexDynDesc._fields_]
