"""CPU-side checks of the boundary: the library loads, exports every entry point
declared in include/*.h, reports errors through status codes, and the Python
mirror validates like the reference (config.rs:54-61)."""
import ctypes as C
import importlib
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in ("hl.h", "hl_debug.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"HL_API\s+[\w\s\*]+?\b(hl_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ["hl_create", "hl_apply_batch", "hl_get_partition", "hl_modularity", "hl_destroy",
                 "hl_num_levels", "hl_last_error", "hl_dbg_move_eval"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    L = importlib.import_module("hit-leiden_b200._lib")
    for name in declared_symbols():
        assert hasattr(L.lib, name), f"libhl.so does not export {name}"


def test_version_and_default_config():
    L = importlib.import_module("hit-leiden_b200._lib")
    assert b"sm_100a" in L.lib.hl_version()
    c = L.Config()
    assert L.lib.hl_config_default(C.byref(c)) == 0
    assert c.resolution == 1.0 and c.mode == 1 and c.max_levels == 10 and c.max_rounds == 20
    assert L.lib.hl_config_default(None) == L.HL_ERR_INVALID_INPUT


def test_null_arguments_return_invalid_input():
    L = importlib.import_module("hit-leiden_b200._lib")
    assert L.lib.hl_num_nodes(None, None) == L.HL_ERR_INVALID_INPUT
    assert b"NULL" in L.lib.hl_last_error()
    L.lib.hl_destroy(None)  # no-op


def test_config_validation_mirrors_reference():
    hl = importlib.import_module("hit-leiden_b200")
    with pytest.raises(hl.HitLeidenError) as e:
        hl.RunConfig(max_iterations=0).validate()
    assert e.value.kind == "InvalidInput"
    with pytest.raises(hl.HitLeidenError):
        hl.RunConfig(quality_tolerance=-1.0).validate()
    hl.RunConfig().validate()


def test_graph_input_arrays():
    hl = importlib.import_module("hit-leiden_b200")
    g = hl.GraphInput("t", 4, [(0, 1, None), (2, 3, 2.5)])
    s, d, w = g.arrays()
    assert s.tolist() == [0, 2] and d.tolist() == [1, 3] and w.tolist() == [1.0, 2.5]
    s, d, w = hl.GraphInput("t", 4, [(0, 1, None)]).arrays()
    assert w is None
