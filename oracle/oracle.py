"""ctypes bindings for the CPU oracle (test infrastructure only).

The oracle restates the reference crate's incremental path in C++
(``oracle/hl_oracle.cpp``).  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this module; the product package never
does.  ``load()`` builds the shared library with ``make`` if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhl_oracle.so")

MODE_DETERMINISTIC = 0
MODE_THROUGHPUT = 1
MAP_F, MAP_G, MAP_S_PRE, MAP_S_CUR, MAP_NODE_TO_COMM = 0, 1, 2, 3, 4
FLAG_KEEP_SELF_LOOPS = 1 << 0
FLAG_AGG_CHANGED_ONLY = 1 << 1
FLAG_EDGE_WEIGHT_LOOPS = 1 << 2
FLAG_NO_COMPACT = 1 << 3
FLAG_FAITHFUL_SCANS = 1 << 4
FLAG_MULTILEVEL = 1 << 5
FLAG_HUB_CHECK = 1 << 6

_lock = threading.Lock()
_lib = None

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("moves", C.c_uint64), ("candidates", C.c_uint64),
                ("traversed", C.c_uint64), ("splits", C.c_uint64), ("merges", C.c_uint64),
                ("changed", C.c_uint64), ("refined", C.c_uint64)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def load():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        src = os.path.join(HERE, "hl_oracle.cpp")
        if (not os.path.exists(LIB_PATH)
                or os.path.getmtime(LIB_PATH) < os.path.getmtime(src)):
            build()
        lib = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        lib.or_graph_from_edges.restype = vp
        lib.or_graph_from_edges.argtypes = [C.c_uint32, u32p, u32p, vp, C.c_uint64]
        lib.or_graph_free.argtypes = [vp]
        lib.or_graph_nodes.restype = C.c_uint32
        lib.or_graph_nodes.argtypes = [vp]
        lib.or_graph_entries.restype = C.c_uint64
        lib.or_graph_entries.argtypes = [vp]
        lib.or_graph_csr.argtypes = [vp, u64p, u32p, f64p]
        lib.or_graph_apply_delta.restype = vp
        lib.or_graph_apply_delta.argtypes = [vp, C.c_uint32, u32p, u32p, vp, C.c_uint64, C.c_int]
        lib.or_node_degrees.argtypes = [vp, f64p]
        lib.or_twice_total_weight.restype = C.c_double
        lib.or_twice_total_weight.argtypes = [vp]
        lib.or_tree_sum.restype = C.c_double
        lib.or_tree_sum.argtypes = [f64p, C.c_uint64]
        lib.or_modularity_edges.restype = C.c_double
        lib.or_modularity_edges.argtypes = [C.c_uint32, u32p, u32p, vp, C.c_uint64, u32p]
        lib.or_modularity_csr.restype = C.c_double
        lib.or_modularity_csr.argtypes = [vp, u32p]
        lib.or_canonicalize.argtypes = [u32p, C.c_uint64]
        lib.or_select_decoupled.restype = C.c_uint64
        lib.or_select_decoupled.argtypes = [u32p, u32p, u32p, vp, f64p, C.c_uint64, u32p]
        lib.or_move_eval.argtypes = [vp, u32p, f64p, C.c_uint64, f64p, C.c_double, C.c_double,
                                     u32p, C.c_uint64, u32p, f64p]
        lib.or_hub_check_counters.argtypes = [u64p]
        lib.or_hub_check_selftest.restype = C.c_int
        lib.or_inc_movement.restype = C.c_uint32
        lib.or_inc_movement.argtypes = [vp, u32p, u32p, vp, C.c_uint64, u32p, u32p, C.c_double,
                                        C.c_int, C.c_uint32, C.c_int, C.c_int, u8p, u8p]
        lib.or_inc_refinement.argtypes = [vp, u32p, u32p, u8p, C.c_double, C.c_int, C.c_int, C.c_int,
                                          u8p]
        lib.or_inc_aggregation.restype = C.c_uint64
        lib.or_inc_aggregation.argtypes = [vp, u32p, u32p, vp, C.c_uint64, u32p, u32p, u8p,
                                           C.c_uint32, u32p, C.POINTER(C.c_uint32), u32p, u32p,
                                           f64p, C.c_uint64]
        lib.or_def_update.argtypes = [C.c_uint32, u32p, u32p, u32p, u8p]
        lib.or_state_new.restype = vp
        lib.or_state_new.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_int, C.c_uint32,
                                     C.c_uint32]
        lib.or_state_free.argtypes = [vp]
        lib.or_state_push_empty_graph.argtypes = [vp, C.c_uint32]
        lib.or_hit_leiden.restype = C.c_int
        lib.or_hit_leiden.argtypes = [vp, C.c_uint32, u32p, u32p, vp, C.c_uint64,
                                      C.POINTER(Stats)]
        lib.or_state_bootstrap.restype = C.c_int
        lib.or_state_bootstrap.argtypes = [vp, C.c_uint32, u32p, u32p, vp, C.c_uint64, C.c_uint32,
                                           C.POINTER(Stats)]
        lib.or_state_import_begin.argtypes = [vp, C.c_uint32, C.c_uint32]
        lib.or_state_import_level.restype = C.c_int
        lib.or_state_import_level.argtypes = [vp, C.c_uint32, C.c_uint32, u64p, u32p, f64p, u32p,
                                              u32p, u32p, u32p]
        lib.or_state_levels.restype = C.c_uint32
        lib.or_state_levels.argtypes = [vp]
        lib.or_state_level_nodes.restype = C.c_uint32
        lib.or_state_level_nodes.argtypes = [vp, C.c_uint32, C.c_int]
        lib.or_state_get_map.restype = C.c_int
        lib.or_state_get_map.argtypes = [vp, C.c_uint32, C.c_int, u32p]
        lib.or_state_set_map.restype = C.c_int
        lib.or_state_set_map.argtypes = [vp, C.c_uint32, C.c_int, u32p, C.c_uint32]
        lib.or_state_graph.restype = vp
        lib.or_state_graph.argtypes = [vp, C.c_uint32]
        lib.or_state_modularity.restype = C.c_double
        lib.or_state_modularity.argtypes = [vp, C.c_uint32, C.c_int]
        lib.or_run.restype = C.c_double
        lib.or_run.argtypes = [C.c_uint32, u32p, u32p, vp, C.c_uint64, C.c_double, C.c_uint32,
                               C.c_uint64, u32p, C.POINTER(C.c_uint32)]
        lib.or_num_threads.restype = C.c_int
        lib.or_num_threads.argtypes = []
        lib.or_set_num_threads.restype = None
        lib.or_set_num_threads.argtypes = [C.c_int]
        _lib = lib
        return lib


def num_threads():
    """Host threads of the throughput mode's snapshot evaluations."""
    return int(load().or_num_threads())


def set_num_threads(threads):
    """Set them (0 = hardware concurrency, at most 64)."""
    load().or_set_num_threads(int(threads))


def _edges(src, dst, w):
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    if w is None:
        return src, dst, None, None
    w = np.ascontiguousarray(w, dtype=np.float64)
    return src, dst, w, w.ctypes.data_as(C.c_void_p)


class Graph:
    """Canonical CSR (rows sorted by neighbour id) held by the oracle."""

    def __init__(self, handle, owned=True):
        self.h = handle
        self.owned = owned

    @classmethod
    def from_edges(cls, n, src, dst, w=None):
        lib = load()
        s, d, wa, wp = _edges(src, dst, w)
        h = lib.or_graph_from_edges(n, s, d, wp, len(s))
        if not h:
            raise ValueError("edge endpoint exceeds node_count")
        return cls(h)

    def __del__(self):
        if getattr(self, "owned", False) and self.h and _lib is not None:
            _lib.or_graph_free(self.h)
            self.h = None

    @property
    def n(self):
        return load().or_graph_nodes(self.h)

    def csr(self):
        lib = load()
        n = self.n
        nnz = lib.or_graph_entries(self.h)
        off = np.zeros(n + 1, np.uint64)
        col = np.zeros(nnz, np.uint32)
        w = np.zeros(nnz, np.float64)
        lib.or_graph_csr(self.h, off, col, w)
        return off, col, w

    def neighbors(self, v):
        off, col, w = self.csr()
        a, b = int(off[v]), int(off[v + 1])
        return list(zip(col[a:b].tolist(), w[a:b].tolist()))

    def total_weight(self):
        return load().or_twice_total_weight(self.h) / 2.0

    def degrees(self):
        out = np.zeros(self.n, np.float64)
        load().or_node_degrees(self.h, out)
        return out

    def apply_delta(self, src, dst, w=None, delta_n=None, keep_self_loops=False):
        lib = load()
        s, d, wa, wp = _edges(src, dst, w)
        dn = self.n if delta_n is None else delta_n
        return Graph(lib.or_graph_apply_delta(self.h, dn, s, d, wp, len(s), int(keep_self_loops)))


def hub_check_counters():
    """Counters of the round-to-round hub key-sum check (FLAG_HUB_CHECK),
    reset by the call: evaluations, mismatches, first-position rescans,
    corrections, table builds, keys scanned."""
    out = np.zeros(6, np.uint64)
    load().or_hub_check_counters(out)
    return dict(zip(("evals", "mismatches", "rescans", "corrections", "builds", "keys"),
                    (int(x) for x in out)))


def hub_check_selftest():
    """The check's stale first-position path on its fixed case: rescans made
    (1 expected), or -1 if an evaluation differed from the full one."""
    return int(load().or_hub_check_selftest())


def tree_sum(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    return load().or_tree_sum(x, len(x))


def modularity_edges(n, src, dst, w, part):
    s, d, wa, wp = _edges(src, dst, w)
    part = np.ascontiguousarray(part, dtype=np.uint32)
    return load().or_modularity_edges(n, s, d, wp, len(s), part)


def modularity_csr(graph: Graph, part):
    return load().or_modularity_csr(graph.h, np.ascontiguousarray(part, dtype=np.uint32))


def canonicalize(c):
    c = np.array(c, dtype=np.uint32)
    load().or_canonicalize(c, len(c))
    return c


def select_decoupled(node, frm, to, gain, kdeg=None):
    node = np.ascontiguousarray(node, np.uint32)
    frm = np.ascontiguousarray(frm, np.uint32)
    to = np.ascontiguousarray(to, np.uint32)
    gain = np.ascontiguousarray(gain, np.float64)
    out = np.zeros(max(1, len(node)), np.uint32)
    kp = None
    if kdeg is not None:
        kdeg = np.ascontiguousarray(kdeg, np.float64)
        kp = kdeg.ctypes.data_as(C.c_void_p)
    cnt = load().or_select_decoupled(node, frm, to, kp, gain, len(node), out)
    return out[:cnt]


def move_eval(graph: Graph, f, d, k, tw, gamma, verts):
    f = np.ascontiguousarray(f, np.uint32)
    d = np.ascontiguousarray(d, np.float64)
    k = np.ascontiguousarray(k, np.float64)
    verts = np.ascontiguousarray(verts, np.uint32)
    to = np.zeros(len(verts), np.uint32)
    gain = np.zeros(len(verts), np.float64)
    load().or_move_eval(graph.h, f, d, len(d), k, tw, gamma, verts, len(verts), to, gain)
    return to, gain


def inc_movement(graph: Graph, dsrc, ddst, dw, f, s, gamma, mode, max_rounds=20, compact=True,
                 mark_moved=False):
    n = graph.n
    ds, dd, dwa, dwp = _edges(dsrc, ddst, dw)
    f = np.array(f, dtype=np.uint32)
    s = np.ascontiguousarray(s, dtype=np.uint32)
    changed = np.zeros(n, np.uint8)
    affected = np.zeros(n, np.uint8)
    it = load().or_inc_movement(graph.h, ds, dd, dwp, len(ds), f, s, gamma, mode, max_rounds,
                                int(compact), int(mark_moved), changed, affected)
    return f, changed.astype(bool), affected.astype(bool), it


def inc_refinement(graph: Graph, f, s, affected, gamma, mode, faithful=False,
                   cc_same_community=False):
    n = graph.n
    f = np.ascontiguousarray(f, dtype=np.uint32)
    s = np.array(s, dtype=np.uint32)
    aff = np.ascontiguousarray(np.asarray(affected, dtype=np.uint8))
    refined = np.zeros(n, np.uint8)
    load().or_inc_refinement(graph.h, f, s, aff, gamma, mode, int(faithful),
                             int(cc_same_community), refined)
    return s, refined.astype(bool)


def inc_aggregation(graph: Graph, dsrc, ddst, dw, s_pre, s_cur, refined, flags=0):
    n = graph.n
    ds, dd, dwa, dwp = _edges(dsrc, ddst, dw)
    s_pre = np.ascontiguousarray(s_pre, np.uint32)
    s_cur = np.ascontiguousarray(s_cur, np.uint32)
    ref = np.ascontiguousarray(np.asarray(refined, dtype=np.uint8))
    nsp = np.zeros(n, np.uint32)
    nn = C.c_uint32(0)
    cap = 4 * (len(ds) + 2 * int(load().or_graph_entries(graph.h)) + 4 * n + 16)
    u = np.zeros(cap, np.uint32)
    v = np.zeros(cap, np.uint32)
    w = np.zeros(cap, np.float64)
    cnt = load().or_inc_aggregation(graph.h, ds, dd, dwp, len(ds), s_pre, s_cur, ref, flags, nsp,
                                    C.byref(nn), u, v, w, cap)
    return (u[:cnt], v[:cnt], w[:cnt]), nsp, nn.value


def def_update(f_levels, s_levels, changed_levels):
    P = len(f_levels)
    sizes = np.array([len(x) for x in f_levels], np.uint32)
    f = np.concatenate([np.asarray(x, np.uint32) for x in f_levels]).astype(np.uint32)
    s = np.concatenate([np.asarray(x, np.uint32) for x in s_levels]).astype(np.uint32)
    ch = np.concatenate([np.asarray(x, np.uint8) for x in changed_levels]).astype(np.uint8)
    load().or_def_update(P, sizes, f, s, ch)
    out_f, out_c, o = [], [], 0
    for p in range(P):
        out_f.append(f[o:o + sizes[p]].copy())
        out_c.append(ch[o:o + sizes[p]].astype(bool))
        o += sizes[p]
    return out_f, out_c


class State:
    """Hierarchical partition state (reference ``PartitionState``, state.rs:19-49)."""

    def __init__(self, n, levels=1, gamma=1.0, mode=MODE_THROUGHPUT, flags=0, max_rounds=20):
        self.lib = load()
        self.h = self.lib.or_state_new(n, levels, gamma, mode, flags, max_rounds)
        self.n = n

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_state_free(self.h)
            self.h = None

    def push_empty_graph(self, n=None):
        self.lib.or_state_push_empty_graph(self.h, self.n if n is None else n)

    def hit_leiden(self, src, dst, w=None, delta_n=None):
        s, d, wa, wp = _edges(src, dst, w)
        st = Stats()
        self.lib.or_hit_leiden(self.h, self.n if delta_n is None else delta_n, s, d, wp, len(s),
                               C.byref(st))
        return st

    def bootstrap(self, src, dst, w=None, max_levels=10):
        s, d, wa, wp = _edges(src, dst, w)
        st = Stats()
        self.lib.or_state_bootstrap(self.h, self.n, s, d, wp, len(s), max_levels, C.byref(st))
        return st

    @property
    def levels(self):
        return self.lib.or_state_levels(self.h)

    def import_levels(self, levels, flags=None):
        """levels: list of dicts with off, col, w, f, g, s_pre, s_cur arrays."""
        fl = (FLAG_MULTILEVEL if len(levels) > 1 else 0) if flags is None else flags
        self.lib.or_state_import_begin(self.h, len(levels), fl)
        for p, lv in enumerate(levels):
            n = len(lv["f"])
            a = [np.ascontiguousarray(lv[k], dt) for k, dt in
                 (("off", np.uint64), ("col", np.uint32), ("w", np.float64), ("f", np.uint32),
                  ("g", np.uint32), ("s_pre", np.uint32), ("s_cur", np.uint32))]
            self.lib.or_state_import_level(self.h, p, n, *a)

    def get_map(self, level, which):
        n = self.lib.or_state_level_nodes(self.h, level, which)
        out = np.zeros(n, np.uint32)
        self.lib.or_state_get_map(self.h, level, which, out)
        return out

    def set_map(self, level, which, arr):
        arr = np.ascontiguousarray(arr, np.uint32)
        self.lib.or_state_set_map(self.h, level, which, arr, len(arr))

    def graph(self, level=0):
        h = self.lib.or_state_graph(self.h, level)
        return Graph(h, owned=False) if h else None

    def modularity(self, level=0, which=MAP_F):
        return self.lib.or_state_modularity(self.h, level, which)


def run(n, src, dst, w=None, gamma=1.0, max_levels=10, seed=42):
    s, d, wa, wp = _edges(src, dst, w)
    part = np.zeros(n, np.uint32)
    lv = C.c_uint32(0)
    q = load().or_run(n, s, d, wp, len(s), gamma, max_levels, seed, part, C.byref(lv))
    return part, q, lv.value
