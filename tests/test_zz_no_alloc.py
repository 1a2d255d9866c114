"""The allocation-free 2m reduction (hl_tree_sum_noalloc).

Some callers cannot let the library allocate device memory: an embedding
runtime that owns every device buffer and hands the library only inputs and
outputs, or code running where cudaMalloc is not allowed.  hl_tree_sum_noalloc
serves them with a fixed scratch array compiled into the library.  This file is
collected last so that a failure here does not hide the other GPU tests; it
must also pass when run alone in a fresh process.

Checked through the C ABI: two calls in a row on caller-owned device buffers
give, bit for bit, the same value as the allocating entry point
(hl_dbg_tree_sum) — the tolerance is exact equality, as for every 2m value —
and sizes above the limit are rejected without touching the GPU.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _allocating_sum(L, x):
    out = C.c_double()
    L.check(L.lib.hl_dbg_tree_sum(0, L.ptr(x), len(x), C.byref(out)))
    return out.value


def test_tree_sum_noalloc_matches_allocating_entry_point_twice():
    import torch

    L = importlib.import_module("hit-leiden_b200._lib")
    torch.cuda.set_device(0)
    rng = np.random.default_rng(2024)
    # several reduction levels, a two-tile case, then the single-tile path
    # (one value, a full tile) and the empty input, which must give +0.0
    sizes = [3_000_001, 1025, 1, 1024, 0]
    for call, n in enumerate(sizes):
        x = rng.uniform(0.1, 3.0, n)
        d_x = torch.from_numpy(x).to("cuda:0") if n else None
        d_out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        st = L.lib.hl_tree_sum_noalloc(C.c_void_p(d_x.data_ptr()) if n else None, n,
                                       C.c_void_p(d_out.data_ptr()), None)
        assert st == L.HL_OK, L.lib.hl_last_error()
        torch.cuda.synchronize()
        got = float(d_out.cpu().numpy()[0])
        want = _allocating_sum(L, x)
        assert np.array_equal(np.array([got]).view(np.uint64), np.array([want]).view(np.uint64)), (
            call, got, want)
        if n == 0:
            assert np.array([got]).view(np.uint64)[0] == 0, got  # +0.0, not -0.0


def test_tree_sum_noalloc_rejects_oversized_input():
    import torch

    L = importlib.import_module("hit-leiden_b200._lib")
    buf = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    ptr = C.c_void_p(buf.data_ptr())  # the size check rejects the call before any launch
    st = L.lib.hl_tree_sum_noalloc(ptr, L.HL_NOALLOC_MAX_ELEMS + 1, ptr, None)
    assert st == L.HL_ERR_INVALID_INPUT
    assert b"exceed" in L.lib.hl_last_error()
