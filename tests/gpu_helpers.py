"""Thin wrappers over libhl's function-level entry points (include/hl_debug.h)
and shared generators for the GPU parity tests."""
from __future__ import annotations

import contextlib
import ctypes as C
import importlib

import numpy as np

from oracle import oracle as O

hl = importlib.import_module("hit-leiden_b200")
L = importlib.import_module("hit-leiden_b200._lib")


def csr_of(g: O.Graph):
    off, col, w = g.csr()
    return g.n, off, col, w


def move_eval(g: O.Graph, f, d, k, tw, gamma, verts):
    n, off, col, w = csr_of(g)
    f, d, k, verts = L.u32(f), L.f64(d), L.f64(k), L.u32(verts)
    to = np.zeros(len(verts), np.uint32)
    gain = np.zeros(len(verts), np.float64)
    L.check(L.lib.hl_dbg_move_eval(0, n, L.ptr(off), L.ptr(col), L.ptr(w), L.ptr(f), L.ptr(d),
                                   len(d), L.ptr(k), tw, gamma, L.ptr(verts), len(verts),
                                   L.ptr(to), L.ptr(gain)))
    return to, gain


def select_decoupled(node, frm, to, gain):
    node, frm, to, gain = L.u32(node), L.u32(frm), L.u32(to), L.f64(gain)
    out = np.zeros(max(1, len(node)), np.uint32)
    cnt = C.c_uint64()
    L.check(L.lib.hl_dbg_select_decoupled(0, L.ptr(node), L.ptr(frm), L.ptr(to), L.ptr(gain),
                                          len(node), L.ptr(out), C.byref(cnt)))
    return out[:cnt.value]


def apply_delta(g: O.Graph, src, dst, w, keep_loops=False, delta_n=None):
    n, off, col, ww = csr_of(g)
    src, dst, w = L.u32(src), L.u32(dst), L.f64(w)
    dn = n if delta_n is None else delta_n
    nn = max(n, dn)
    cap = len(col) + 2 * len(src) + 2
    ooff = np.zeros(nn + 1, np.uint64)
    ocol = np.zeros(cap, np.uint32)
    ow = np.zeros(cap, np.float64)
    nnz = C.c_uint64()
    L.check(L.lib.hl_dbg_apply_delta(0, n, L.ptr(off), L.ptr(col), L.ptr(ww), dn, L.ptr(src),
                                     L.ptr(dst), L.ptr(w), len(src), int(keep_loops), L.ptr(ooff),
                                     L.ptr(ocol), L.ptr(ow), cap, C.byref(nnz)))
    return ooff, ocol[:nnz.value], ow[:nnz.value]


def inc_movement(g: O.Graph, dsrc, ddst, dw, f, s, gamma, max_rounds=20, mark_moved=False):
    n, off, col, w = csr_of(g)
    dsrc, ddst, dw = L.u32(dsrc), L.u32(ddst), L.f64(dw)
    f = np.array(f, dtype=np.uint32)
    s = L.u32(s)
    ch = np.zeros(n, np.uint8)
    af = np.zeros(n, np.uint8)
    it = C.c_uint32()
    L.check(L.lib.hl_dbg_inc_movement(0, n, L.ptr(off), L.ptr(col), L.ptr(w), L.ptr(dsrc),
                                      L.ptr(ddst), L.ptr(dw), len(dsrc), L.ptr(f), L.ptr(s), gamma,
                                      max_rounds, int(mark_moved), L.ptr(ch), L.ptr(af),
                                      C.byref(it)))
    return f, ch.astype(bool), af.astype(bool), it.value


@contextlib.contextmanager
def exact_tfilter(on=True):
    """Make the T-filter decide every candidate from the ordered sum."""
    L.check(L.lib.hl_dbg_set_exact_tfilter(int(on)))
    try:
        yield
    finally:
        L.check(L.lib.hl_dbg_set_exact_tfilter(0))


@contextlib.contextmanager
def bucket_slots(slots):
    """Shrink the partitioned hub pass's tables (0 = default) for a block."""
    L.check(L.lib.hl_dbg_set_bucket_slots(int(slots)))
    try:
        yield
    finally:
        L.check(L.lib.hl_dbg_set_bucket_slots(0))


@contextlib.contextmanager
def hub_defer(entries):
    """Send integral hub rows longer than `entries` straight to the
    partitioned pass (0 = default) for a block."""
    L.check(L.lib.hl_dbg_set_hub_defer(int(entries)))
    try:
        yield
    finally:
        L.check(L.lib.hl_dbg_set_hub_defer(0))


@contextlib.contextmanager
def bins(mid_max, wide_max):
    """Warp-bin thresholds of the stage entry points for a block."""
    L.check(L.lib.hl_dbg_set_bins(int(mid_max), int(wide_max)))
    try:
        yield
    finally:
        L.check(L.lib.hl_dbg_set_bins(0, 0))


@contextlib.contextmanager
def stage_mode(mode):
    """Run the stage entry points in `mode` (hl.RunMode), throughput after."""
    L.check(L.lib.hl_dbg_set_mode(int(mode)))
    try:
        yield
    finally:
        L.check(L.lib.hl_dbg_set_mode(L.HL_MODE_THROUGHPUT))


def inc_refinement(g: O.Graph, f, s, affected, gamma, cc_same_community=False):
    n, off, col, w = csr_of(g)
    f = L.u32(f)
    s = np.array(s, dtype=np.uint32)
    aff = np.ascontiguousarray(np.asarray(affected, dtype=np.uint8))
    ref = np.zeros(n, np.uint8)
    L.check(L.lib.hl_dbg_inc_refinement(0, n, L.ptr(off), L.ptr(col), L.ptr(w), L.ptr(f),
                                        L.ptr(s), L.ptr(aff), gamma, int(cc_same_community),
                                        L.ptr(ref)))
    return s, ref.astype(bool)


def inc_aggregation(g: O.Graph, dsrc, ddst, dw, s_pre, s_cur, refined, changed_only=False,
                    edge_weight_loops=False):
    n, off, col, w = csr_of(g)
    dsrc, ddst, dw = L.u32(dsrc), L.u32(ddst), L.f64(dw)
    s_pre, s_cur = L.u32(s_pre), L.u32(s_cur)
    ref = np.ascontiguousarray(np.asarray(refined, dtype=np.uint8))
    cap = 4 * (len(dsrc) + len(col) + 2 * n + 8)
    ou = np.zeros(cap, np.uint32)
    ov = np.zeros(cap, np.uint32)
    ow = np.zeros(cap, np.float64)
    nsp = np.zeros(n, np.uint32)
    nn = C.c_uint32()
    cnt = C.c_uint64()
    L.check(L.lib.hl_dbg_inc_aggregation(0, n, L.ptr(off), L.ptr(col), L.ptr(w), L.ptr(dsrc),
                                         L.ptr(ddst), L.ptr(dw), len(dsrc), L.ptr(s_pre),
                                         L.ptr(s_cur), L.ptr(ref), int(changed_only),
                                         int(edge_weight_loops), L.ptr(nsp), C.byref(nn),
                                         L.ptr(ou), L.ptr(ov), L.ptr(ow), cap, C.byref(cnt)))
    c = cnt.value
    return (ou[:c], ov[:c], ow[:c]), nsp, nn.value


def tree_sum(x):
    x = L.f64(x)
    out = C.c_double()
    L.check(L.lib.hl_dbg_tree_sum(0, L.ptr(x), len(x), C.byref(out)))
    return out.value


def modularity(g: O.Graph, part):
    n, off, col, w = csr_of(g)
    part = L.u32(part)
    q = C.c_double()
    L.check(L.lib.hl_dbg_modularity(0, n, L.ptr(off), L.ptr(col), L.ptr(w), L.ptr(part),
                                    C.byref(q)))
    return q.value


# ---------------------------------------------------------------------------
def random_graph(rng, n, m, integral=True, loops=0.0):
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    if loops <= 0.0:
        keep = src != dst
        src, dst = src[keep], dst[keep]
    if integral:
        w = rng.integers(1, 4, len(src)).astype(np.float64)
    else:
        w = rng.uniform(0.5, 2.0, len(src))
    return src.astype(np.uint32), dst.astype(np.uint32), w


def random_partition(rng, n, k):
    return rng.integers(0, k, n).astype(np.uint32)


def same_bits(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype == np.float64:
        return np.array_equal(a.view(np.uint64), b.view(np.uint64))
    return np.array_equal(a, b)
