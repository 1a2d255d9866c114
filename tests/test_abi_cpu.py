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
    # RunConfig::default() (config.rs:37-48): deterministic mode, 10 iterations
    assert c.resolution == 1.0 and c.mode == L.HL_MODE_DETERMINISTIC
    assert c.max_levels == 10 and c.max_rounds == 20
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
    assert hl.RunConfig().mode == hl.RunMode.Deterministic


def test_graph_input_arrays():
    hl = importlib.import_module("hit-leiden_b200")
    g = hl.GraphInput("t", 4, [(0, 1, None), (2, 3, 2.5)])
    s, d, w = g.arrays()
    assert s.tolist() == [0, 2] and d.tolist() == [1, 3] and w.tolist() == [1.0, 2.5]
    s, d, w = hl.GraphInput("t", 4, [(0, 1, None)]).arrays()
    assert w is None


def test_struct_layouts_match_the_header(tmp_path):
    # the ctypes mirrors must have the C header's sizes and field offsets:
    # a small C program compiled against include/hl.h prints them
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    L = importlib.import_module("hit-leiden_b200._lib")
    structs = {"hl_config": L.Config, "hl_batch_stats": L.BatchStats,
               "hl_request_done": L.RequestDone, "hl_kernel_stat": L.KernelStat}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "hl.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            parts = line.split()
            got[(parts[0], parts[1])] = int(parts[2])
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_graph_input_widens_f32_weights_exactly():
    import numpy as np
    hl = importlib.import_module("hit-leiden_b200")
    w32 = np.array([0.1, 1.5, 3.25, 1e-7], np.float32)
    g = hl.GraphInput.from_arrays("t", 5, [0, 1, 2, 3], [1, 2, 3, 4], w32)
    src, dst, w = g.arrays()
    assert w.dtype == np.float64 and np.array_equal(w, w32.astype(np.float64))
    assert src.dtype == np.uint32 and dst.dtype == np.uint32


def test_library_exports_no_undeclared_entry_points():
    # every hl_* symbol the library exports is declared in include/*.h (the
    # build hides everything else of its own)
    import shutil
    import subprocess
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("no nm")
    lib = os.path.join(ROOT, "hit-leiden_b200", "libhl.so")
    out = subprocess.run([nm, "-D", "--defined-only", lib], check=True, capture_output=True,
                         text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.split()[-1].startswith("hl_")}
    assert exported == set(declared_symbols())


def test_rust_binding_mirrors_the_header():
    """rust/hit-leiden-gpu/src/ffi.rs declares every entry point of
    include/hl.h, and its #[repr(C)] structs have the header's fields in the
    header's order (the crate is not compiled in this image: no cargo)."""
    ffi = open(os.path.join(ROOT, "rust", "hit-leiden-gpu", "src", "ffi.rs")).read()
    text = open(os.path.join(ROOT, "include", "hl.h")).read()
    public = sorted(set(re.findall(r"HL_API\s+[\w\s\*]+?\b(hl_\w+)\s*\(", text)))
    for name in public:
        assert re.search(rf"pub fn {name}\s*\(", ffi), f"ffi.rs lacks {name}"
    for cname in ("hl_config", "hl_batch_stats", "hl_kernel_stat", "hl_request_done"):
        body_c = re.search(r"typedef struct \{([^{}]*)\}\s*" + cname + ";", text).group(1)
        fields_c = re.findall(r"\b(\w+)(?:\[\d+\])?;", re.sub(r"/\*.*?\*/", "", body_c, flags=re.S))
        body_r = re.search(r"pub struct " + cname + r" \{(.*?)\}", ffi, re.S).group(1)
        fields_r = re.findall(r"pub (\w+):", body_r)
        assert fields_c == fields_r, (cname, fields_c, fields_r)
