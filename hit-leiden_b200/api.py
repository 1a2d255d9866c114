"""Python mirror of the reference crate's API for the incremental update path.

Names, argument meaning and errors follow the Rust crate ``hit_leiden`` 0.1.0:

* ``GraphInput`` (src/core/types.rs:133-147): node_count + edge list; a ``None``
  weight means 1.0, a negative weight weakens or deletes an edge.
* ``RunConfig`` / ``RunMode`` (src/core/config.rs:19-63) and ``validate()``.
* ``PartitionState`` (src/core/partition/state.rs:19-49): here the state lives
  on the GPU behind a libhl handle; the per-level vectors are read back on access.
* ``hit_leiden(state, delta, gamma, mode)`` (hit_leiden.rs:936-1018) returns the
  number of movement iterations.
* ``run(graph, config)`` (lib.rs:27-29 → hit_leiden.rs:30-118) loads a graph,
  builds the hierarchy and returns a ``RunOutcome`` with a ``PartitionResult``.
* ``HitLeidenError`` with ``kind == "InvalidInput"`` for the cases the reference
  rejects (config.rs:54-61, hit_leiden.rs:35-43).

Every computation runs in libhl.so on the GPU; nothing here computes partitions.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L
from ._lib import HitLeidenError


class RunMode(enum.IntEnum):
    """RunMode (config.rs:19-23).  Both modes run on the GPU: Deterministic is
    the sequential Gauss–Seidel form (the reference's default), Throughput the
    round-based parallel form and the fast path."""
    Deterministic = 0
    Throughput = 1
    DETERMINISTIC = 0
    THROUGHPUT = 1


@dataclass
class RunConfig:
    """RunConfig (config.rs:25-63).  ``max_iterations`` caps the hierarchy
    levels exactly as it caps multilevel_leiden's levels (hit_leiden.rs:217);
    1 reproduces the reference's single-level PartitionState (state.rs:42).
    The defaults are RunConfig::default() (config.rs:37-48): deterministic
    mode, 10 iterations, resolution 1.0, tolerance 0.001."""
    mode: RunMode = RunMode.Deterministic
    resolution: float = 1.0
    max_iterations: int = 10
    quality_tolerance: float = 0.001
    max_rounds: int = 20
    device: int = 0
    hbm_budget: int = 0
    keep_self_loops: bool = False
    batch_modularity: bool = False
    kernel_timing: bool = False
    autotune: bool = True        # degree-bin autotuner (HL_FLAG_NO_AUTOTUNE when off)
    small_rounds: bool = True    # one-block rounds for small frontiers (HL_FLAG_NO_SMALL_ROUNDS)

    def validate(self) -> None:
        if self.max_iterations == 0:
            raise HitLeidenError(L.HL_ERR_INVALID_INPUT, "max_iterations must be > 0")
        if self.quality_tolerance < 0.0:
            raise HitLeidenError(L.HL_ERR_INVALID_INPUT, "quality_tolerance must be >= 0")

    def to_c(self) -> L.Config:
        c = L.Config()
        L.check(L.lib.hl_config_default(C.byref(c)))
        c.resolution = float(self.resolution)
        c.mode = int(self.mode)
        c.max_levels = int(self.max_iterations)
        c.max_rounds = int(self.max_rounds)
        c.flags = ((L.HL_FLAG_KEEP_SELF_LOOPS if self.keep_self_loops else 0)
                   | (L.HL_FLAG_BATCH_MODULARITY if self.batch_modularity else 0)
                   | (L.HL_FLAG_KERNEL_TIMING if self.kernel_timing else 0)
                   | (0 if self.autotune else L.HL_FLAG_NO_AUTOTUNE)
                   | (0 if self.small_rounds else L.HL_FLAG_NO_SMALL_ROUNDS))
        c.hbm_budget = int(self.hbm_budget)
        c.device = int(self.device)
        return c


@dataclass
class GraphInput:
    """GraphInput (types.rs:133-147).  Edges may be given as a list of
    (u, v, weight-or-None) tuples or, for large graphs, as arrays."""
    dataset_id: str
    node_count: int
    edges: List[Tuple[int, int, Optional[float]]] = field(default_factory=list)
    _arrays: Optional[Tuple[np.ndarray, np.ndarray, Optional[np.ndarray]]] = None

    @classmethod
    def empty(cls, dataset_id: str = "") -> "GraphInput":
        return cls(dataset_id, 0, [])

    @classmethod
    def from_arrays(cls, dataset_id: str, node_count: int, src, dst, w=None) -> "GraphInput":
        g = cls(dataset_id, node_count, [])
        g._arrays = (L.u32(src), L.u32(dst), L.f64(w))
        return g

    def arrays(self):
        if self._arrays is not None:
            return self._arrays
        m = len(self.edges)
        src = np.fromiter((e[0] for e in self.edges), dtype=np.int64, count=m)
        dst = np.fromiter((e[1] for e in self.edges), dtype=np.int64, count=m)
        if np.any(src < 0) or np.any(dst < 0):
            raise HitLeidenError(L.HL_ERR_INVALID_INPUT, "negative edge endpoint")
        if any(e[2] is not None for e in self.edges):
            w = np.array([1.0 if e[2] is None else float(e[2]) for e in self.edges], np.float64)
        else:
            w = None
        return L.u32(src), L.u32(dst), w

    def __len__(self):
        return len(self._arrays[0]) if self._arrays is not None else len(self.edges)


@dataclass
class PartitionResult:
    """PartitionResult (types.rs:103-113)."""
    run_id: str
    node_to_community: np.ndarray
    hierarchy_levels: List[np.ndarray]
    community_count: int
    quality_score: float
    iteration_count: int


@dataclass
class RunOutcome:
    partition: Optional[PartitionResult]
    state: Optional["PartitionState"] = None


class PartitionState:
    """GPU-resident hierarchical state (state.rs:19-32).

    The reference's public fields are exposed as read-only properties that copy
    the per-level vectors back from the device.
    """

    def __init__(self, handle: C.c_void_p, node_count: int, config: RunConfig):
        self._h = handle
        self._n = node_count
        self.config = config
        self.last_stats: Optional[L.BatchStats] = None

    # -- construction ------------------------------------------------------
    @classmethod
    def load(cls, graph: GraphInput, config: Optional[RunConfig] = None) -> "PartitionState":
        """Load ``graph`` onto the GPU and build the bootstrap partition."""
        config = config or RunConfig()
        config.validate()
        src, dst, w = graph.arrays()
        h = C.c_void_p()
        cfg = config.to_c()
        L.check(L.lib.hl_create(C.byref(cfg), int(graph.node_count), L.ptr(src), L.ptr(dst),
                                L.ptr(w), len(src), C.byref(h)))
        return cls(h, int(graph.node_count), config)

    def close(self) -> None:
        if self._h:
            L.lib.hl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- reference fields --------------------------------------------------
    @property
    def node_count(self) -> int:
        return self._n

    @property
    def levels(self) -> int:
        x = C.c_uint32()
        L.check(L.lib.hl_num_levels(self._h, C.byref(x)))
        return x.value

    def level_size(self, level: int) -> int:
        x = C.c_uint32()
        L.check(L.lib.hl_level_size(self._h, level, C.byref(x)))
        return x.value

    def _map(self, level: int, which: int) -> np.ndarray:
        out = np.zeros(self.level_size(level), np.uint32)
        L.check(L.lib.hl_get_map(self._h, level, which, L.ptr(out)))
        return out

    def _maps(self, which: int) -> List[np.ndarray]:
        return [self._map(p, which) for p in range(self.levels)]

    @property
    def community_mapping_per_level(self) -> List[np.ndarray]:
        return self._maps(L.HL_MAP_COMMUNITY)

    @property
    def refined_community_mapping_per_level(self) -> List[np.ndarray]:
        return self._maps(L.HL_MAP_REFINED)

    @property
    def previous_subcommunity_mapping_per_level(self) -> List[np.ndarray]:
        return self._maps(L.HL_MAP_SUB_PREVIOUS)

    @property
    def current_subcommunity_mapping_per_level(self) -> List[np.ndarray]:
        return self._maps(L.HL_MAP_SUB_CURRENT)

    @property
    def node_to_comm(self) -> np.ndarray:
        """g¹ (hit_leiden.rs:1016): the refined mapping of level 0."""
        return self._map(0, L.HL_MAP_REFINED)

    def supergraph(self, level: int = 0):
        """CSR of G^level: (offsets, neighbours, weights), rows sorted."""
        n = self.level_size(level)
        nnz = C.c_uint64()
        L.check(L.lib.hl_num_edges(self._h, level, C.byref(nnz)))
        off = np.zeros(n + 1, np.uint64)
        col = np.zeros(nnz.value, np.uint32)
        w = np.zeros(nnz.value, np.float64)
        L.check(L.lib.hl_get_csr(self._h, level, L.ptr(off), L.ptr(col), L.ptr(w)))
        return off, col, w

    # -- results -----------------------------------------------------------
    def partition(self) -> np.ndarray:
        """Community of every input vertex, relabelled 0..k-1 first-seen."""
        out = np.zeros(self._n, np.uint32)
        L.check(L.lib.hl_get_partition(self._h, L.ptr(out)))
        return out

    def modularity(self, partition=None) -> float:
        q = C.c_double()
        if partition is None:
            L.check(L.lib.hl_modularity(self._h, C.byref(q)))
        else:
            p = L.u32(partition)
            L.check(L.lib.hl_modularity_of(self._h, L.ptr(p), C.byref(q)))
        return q.value

    def set_level_callback(self, fn) -> None:
        """Per-level output (hl_set_level_callback): during apply_batch,
        ``fn(level, nodes, sub_ids)`` is called after each level's refinement
        with the level's nodes whose sub-community changed in the batch and
        their new ids (numpy copies).  None turns it off."""
        if fn is None:
            self._level_cb = None
            L.check(L.lib.hl_set_level_callback(self._h, L.LEVEL_FN(), None))
            return

        def tramp(user, level, count, nodes, ids):
            nn = np.ctypeslib.as_array(nodes, (count,)).copy() if count else np.zeros(0, np.uint32)
            ii = np.ctypeslib.as_array(ids, (count,)).copy() if count else np.zeros(0, np.uint32)
            fn(int(level), nn, ii)
        self._level_cb = L.LEVEL_FN(tramp)  # kept alive with the state
        L.check(L.lib.hl_set_level_callback(self._h, self._level_cb, None))

    def kernel_stats(self) -> dict:
        """Per-kernel launches, device ms, algorithmic bytes and items since
        creation or the last reset (config.kernel_timing must be set)."""
        kst = (L.KernelStat * 64)()
        cnt = C.c_uint32()
        L.check(L.lib.hl_kernel_stats(self._h, kst, 64, C.byref(cnt)))
        return {kst[i].name.decode(): {"launches": kst[i].launches, "ms": kst[i].total_ms,
                                       "bytes": kst[i].bytes, "items": kst[i].items}
                for i in range(min(cnt.value, 64))}

    def apply_batch(self, src, dst, w=None) -> L.BatchStats:
        src, dst, w = L.u32(src), L.u32(dst), L.f64(w)
        st = L.BatchStats()
        L.check(L.lib.hl_apply_batch(self._h, L.ptr(src), L.ptr(dst), L.ptr(w), len(src),
                                     C.byref(st)))
        self.last_stats = st
        return st


def hit_leiden(state: PartitionState, delta_g: GraphInput, gamma: float = 1.0,
               mode: RunMode = RunMode.Deterministic) -> int:
    """Algorithm 6 (hit_leiden.rs:936-1018): apply ``delta_g`` and update every
    level in ``mode``.  Returns the total number of movement iterations (one
    per level in deterministic mode, as the reference returns)."""
    if int(mode) != int(state.config.mode):
        L.check(L.lib.hl_set_mode(state._h, int(mode)))
        state.config.mode = RunMode(int(mode))
    if gamma != state.config.resolution:
        L.check(L.lib.hl_set_resolution(state._h, float(gamma)))
        state.config.resolution = gamma
    src, dst, w = delta_g.arrays()
    return state.apply_batch(src, dst, w).iterations


# ---------------------------------------------------------------------------
# Many graphs on one GPU (no reference counterpart): batching and serving.
# ---------------------------------------------------------------------------
def apply_batches(states: Sequence[PartitionState], batches, workers: int = 16):
    """Batching form: apply batches[i] = (src, dst, w or None) to states[i] for
    every i at once (hl_apply_batches).  Each state ends exactly as
    ``states[i].apply_batch(*batches[i])`` would leave it; graphs run
    concurrently on their own streams.  Returns the per-graph BatchStats."""
    n = len(states)
    if len(batches) != n:
        raise HitLeidenError(L.HL_ERR_INVALID_INPUT, "one batch per state is required")
    keep = []
    hs = (C.c_void_p * n)()
    ps = (C.c_void_p * n)()
    pd = (C.c_void_p * n)()
    pw = (C.c_void_p * n)()
    ks = (C.c_uint64 * n)()
    for i, (st, b) in enumerate(zip(states, batches)):
        src, dst = L.u32(b[0]), L.u32(b[1])
        w = L.f64(b[2]) if len(b) > 2 else None
        keep.append((src, dst, w))
        hs[i] = st._h.value if isinstance(st._h, C.c_void_p) else st._h
        ps[i] = src.ctypes.data if len(src) else None
        pd[i] = dst.ctypes.data if len(dst) else None
        pw[i] = w.ctypes.data if (w is not None and len(w)) else None
        ks[i] = len(src)
    stats = (L.BatchStats * n)()
    statuses = (C.c_int * n)()
    vp = C.c_void_p
    L.check(L.lib.hl_apply_batches(C.cast(hs, vp), C.cast(ps, vp), C.cast(pd, vp), C.cast(pw, vp),
                                   C.cast(ks, vp), n, int(workers), C.cast(statuses, vp), stats))
    for st, s_ in zip(states, stats):
        st.last_stats = s_
    return list(stats)


class Server:
    """Serving form (hl_server_*): a request loop over resident graphs.

    Requests are admitted against ``hbm_budget`` bytes (0 = unlimited); the
    requests a graph receives while it is being updated are coalesced, in
    arrival order, into its next batch; ``workers`` threads update different
    graphs concurrently.  The server does not own the states: close it first."""

    def __init__(self, workers: int = 8, hbm_budget: int = 0):
        self._s = C.c_void_p()
        L.check(L.lib.hl_server_create(int(workers), int(hbm_budget), C.byref(self._s)))
        self._states = []

    def add(self, state: PartitionState) -> int:
        gid = C.c_uint32()
        L.check(L.lib.hl_server_add_graph(self._s, state._h, C.byref(gid)))
        self._states.append(state)
        return gid.value

    def set_level_callback(self, fn) -> None:
        """Per-level output of the served batches: ``fn(graph, batch_id, level,
        nodes, sub_ids)`` from the worker thread, after each level's
        refinement and before the batch's requests complete.  None turns it
        off.  Set it before submitting."""
        if fn is None:
            self._level_cb = None
            L.check(L.lib.hl_server_set_level_callback(self._s, L.SERVER_LEVEL_FN(), None))
            return

        def tramp(user, graph, batch_id, level, count, nodes, ids):
            nn = np.ctypeslib.as_array(nodes, (count,)).copy() if count else np.zeros(0, np.uint32)
            ii = np.ctypeslib.as_array(ids, (count,)).copy() if count else np.zeros(0, np.uint32)
            fn(int(graph), int(batch_id), int(level), nn, ii)
        self._level_cb = L.SERVER_LEVEL_FN(tramp)
        L.check(L.lib.hl_server_set_level_callback(self._s, self._level_cb, None))

    def set_edge_estimate(self, bytes_per_edge: int) -> None:
        L.check(L.lib.hl_server_set_edge_estimate(self._s, int(bytes_per_edge)))

    def set_coalescing(self, max_requests: int) -> None:
        """At most ``max_requests`` per batch (0 = all pending; 1 = none)."""
        L.check(L.lib.hl_server_set_coalescing(self._s, int(max_requests)))

    def submit(self, graph_id: int, src, dst, w=None) -> int:
        src, dst, w = L.u32(src), L.u32(dst), L.f64(w)
        rid = C.c_uint64()
        L.check(L.lib.hl_server_submit(self._s, int(graph_id), L.ptr(src), L.ptr(dst), L.ptr(w),
                                       len(src), C.byref(rid)))
        return rid.value

    def poll(self, cap: int = 4096, wait_ms: int = 0):
        out = (L.RequestDone * cap)()
        cnt = C.c_uint32()
        L.check(L.lib.hl_server_poll(self._s, out, cap, C.byref(cnt), int(wait_ms)))
        return [out[i].as_dict() for i in range(cnt.value)]

    def drain(self) -> None:
        L.check(L.lib.hl_server_drain(self._s))

    def close(self) -> None:
        if self._s:
            L.lib.hl_server_destroy(self._s)
            self._s = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compute_modularity(graph: GraphInput, node_to_community) -> float:
    """compute_modularity (hit_leiden.rs:121-161) on the GPU."""
    src, dst, w = graph.arrays()
    n = int(graph.node_count)
    # Build the canonical CSR through apply_delta on an empty graph.
    off0 = np.zeros(n + 1, np.uint64)
    cap = 2 * len(src) + 2
    off = np.zeros(n + 1, np.uint64)
    col = np.zeros(cap, np.uint32)
    ww = np.zeros(cap, np.float64)
    nnz = C.c_uint64()
    e = np.zeros(1, np.uint32)
    L.check(L.lib.hl_dbg_apply_delta(0, n, L.ptr(off0), L.ptr(e), None, n, L.ptr(src),
                                     L.ptr(dst), L.ptr(w), len(src), 1, L.ptr(off), L.ptr(col),
                                     L.ptr(ww), cap, C.byref(nnz)))
    part = L.u32(node_to_community)
    q = C.c_double()
    L.check(L.lib.hl_dbg_modularity(0, n, L.ptr(off), L.ptr(col), L.ptr(ww), L.ptr(part),
                                    C.byref(q)))
    return q.value


def canonicalize_community_ids(ids: Sequence[int], device: int = 0) -> np.ndarray:
    """First-seen contiguous relabelling (hit_leiden.rs:358-376) on the GPU."""
    a = np.array(ids, dtype=np.uint32)
    L.check(L.lib.hl_canonicalize(device, L.ptr(a), len(a)))
    return a


def run(graph: GraphInput, config: Optional[RunConfig] = None, keep_state: bool = False
        ) -> RunOutcome:
    """Load + bootstrap on the GPU and return the partition (lib.rs:27-29).

    Validation mirrors hit_leiden.rs:31-43 (config, then endpoints)."""
    config = config or RunConfig()
    config.validate()
    src, dst, w = graph.arrays()
    if len(src) and (int(src.max()) >= graph.node_count or int(dst.max()) >= graph.node_count):
        raise HitLeidenError(L.HL_ERR_INVALID_INPUT, "edge endpoint exceeds node_count")
    st = PartitionState.load(graph, config)
    part = st.partition()
    q = st.modularity()
    levels = []
    subs = st.current_subcommunity_mapping_per_level
    chain = np.arange(graph.node_count, dtype=np.uint32)
    for p in range(st.levels):
        levels.append(canonicalize_community_ids(chain, config.device) if len(chain) else chain)
        if p < len(subs):
            chain = subs[p][chain]
    res = PartitionResult(run_id=f"run:{graph.dataset_id}", node_to_community=part,
                          hierarchy_levels=levels, community_count=int(len(np.unique(part))),
                          quality_score=q, iteration_count=0)
    out = RunOutcome(partition=res, state=st if keep_state else None)
    if not keep_state:
        st.close()
    return out
