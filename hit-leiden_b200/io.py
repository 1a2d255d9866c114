"""Host-side inputs and reports around the update path, in the reference's
conventions.

* Edge-list loading (the reference's loaders, src/main.rs:189-230 and
  src/bin/profile_incremental.rs:32-65): one ``src dst [weight]`` per line
  (README.md:37-38); self-loops are skipped; a symmetric listing (both
  directions present, as webgraph stores them) keeps ``src < dst`` only.
* Batch schedules (src/benchmark/dynamic_graph.rs:54-131): cumulative chunks,
  and the paper split (initial ratio of shuffled edges, then fixed-size
  update rounds).  The shuffle uses numpy's seeded generator; the reference's
  ``rand::StdRng`` permutation is not reproduced, only the split's shape.
* Partition comparison (src/benchmark/hit_leiden_incremental.rs:513-665):
  community sizes, NMI (mutual information over the geometric mean of the
  two entropies, natural log), purity in both directions, and the Jaccard
  index of the two largest communities (largest size, smallest id on ties).

These are plain numpy utilities: the update path itself is libhl.so.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np


# ---------------------------------------------------------------------------
# Loading
# ---------------------------------------------------------------------------
@dataclass
class EdgeList:
    """An undirected edge list: ``node_count`` vertices, SoA ``src, dst, w``."""
    dataset_id: str
    node_count: int
    src: np.ndarray
    dst: np.ndarray
    w: np.ndarray
    self_loops_skipped: int = 0

    def __len__(self) -> int:
        return len(self.src)


def parse_edge_list(text: str, symmetric: bool = False, node_count: Optional[int] = None,
                    dataset_id: str = "edges") -> EdgeList:
    """Parse ``src dst [weight]`` lines.  Blank lines and lines starting with
    ``#`` or ``%`` are comments.  Self-loops are skipped.  With
    ``symmetric=True`` (both directions listed) only ``src < dst`` is kept;
    otherwise every line is one undirected edge, oriented ``(min, max)``.
    A missing weight is 1.0 (in_memory.rs:49)."""
    us, vs, ws = [], [], []
    loops = 0
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line[0] in "#%":
            continue
        parts = line.replace(",", " ").split()
        if len(parts) < 2:
            raise ValueError(f"malformed edge line: {raw!r}")
        u, v = int(parts[0]), int(parts[1])
        if u < 0 or v < 0:
            raise ValueError(f"negative vertex id in line: {raw!r}")
        x = float(parts[2]) if len(parts) > 2 else 1.0
        if u == v:
            loops += 1
            continue
        if symmetric:
            if u > v:
                continue
        elif u > v:
            u, v = v, u
        us.append(u)
        vs.append(v)
        ws.append(x)
    src = np.asarray(us, dtype=np.uint32)
    dst = np.asarray(vs, dtype=np.uint32)
    n = int(max(int(src.max()), int(dst.max())) + 1) if len(src) else 0
    if node_count is not None:
        if node_count < n:
            raise ValueError(f"node_count {node_count} < largest id + 1 ({n})")
        n = node_count
    return EdgeList(dataset_id, n, src, dst, np.asarray(ws, dtype=np.float64), loops)


def load_edge_list(path: str, symmetric: bool = False, node_count: Optional[int] = None
                   ) -> EdgeList:
    """Read a text edge list from ``path`` (see :func:`parse_edge_list`)."""
    import os
    with open(path, "r", encoding="utf-8") as fh:
        text = fh.read()
    stem = os.path.splitext(os.path.basename(path))[0]
    return parse_edge_list(text, symmetric=symmetric, node_count=node_count, dataset_id=stem)


# ---------------------------------------------------------------------------
# Batch schedules
# ---------------------------------------------------------------------------
@dataclass
class IncrementalSplit:
    initial: EdgeList
    updates: List[EdgeList]      # cumulative graph after each update round
    deltas: List[EdgeList]       # the edges each round adds (the update batch)
    batch_size: int
    rounds: int


def _subset(e: EdgeList, idx: np.ndarray, name: str) -> EdgeList:
    return EdgeList(name, e.node_count, e.src[idx], e.dst[idx], e.w[idx])


def cumulative_batches(edges: EdgeList, batch_size: int) -> List[EdgeList]:
    """dynamic_graph.rs:54-72: chunks of ``batch_size`` edges in order; batch
    i holds every edge of chunks 0..i."""
    if batch_size <= 0:
        raise ValueError("batch_size must be positive")
    out = []
    for i, start in enumerate(range(0, len(edges), batch_size)):
        end = min(start + batch_size, len(edges))
        out.append(_subset(edges, np.arange(end), f"batch_{i}"))
    return out


def paper_split(edges: EdgeList, initial_ratio: float, batch_size: int, rounds: int,
                seed: int) -> IncrementalSplit:
    """dynamic_graph.rs:78-131: shuffle, keep floor(ratio·m) edges as the
    initial graph, then ``min(rounds, remaining // batch_size)`` rounds of
    ``batch_size`` edges each (cumulative graphs, plus each round's delta)."""
    m = len(edges)
    perm = np.random.default_rng(seed).permutation(m)
    ratio = min(max(initial_ratio, 0.0), 1.0)
    k0 = int(np.floor(m * ratio))
    avail = m - k0
    eff = 0 if batch_size == 0 else min(rounds, avail // batch_size)
    initial = _subset(edges, perm[:k0], "paper_initial")
    updates, deltas = [], []
    for r in range(eff):
        end = k0 + (r + 1) * batch_size
        updates.append(_subset(edges, perm[:end], f"paper_batch_{r}"))
        deltas.append(_subset(edges, perm[end - batch_size:end], f"paper_delta_{r}"))
    return IncrementalSplit(initial, updates, deltas, batch_size, eff)


# ---------------------------------------------------------------------------
# Partition comparison
# ---------------------------------------------------------------------------
def community_sizes(partition: Sequence[int]) -> dict:
    ids, counts = np.unique(np.asarray(partition), return_counts=True)
    return {int(i): int(c) for i, c in zip(ids, counts)}


def largest_community(partition: Sequence[int]) -> Tuple[int, int]:
    """(id, size) of the largest community; the smallest id on equal sizes
    (hit_leiden_incremental.rs:519-528)."""
    sizes = community_sizes(partition)
    if not sizes:
        return 0, 0
    best = max(sizes.items(), key=lambda kv: (kv[1], -kv[0]))
    return best


def _entropy(counts: np.ndarray, n: float) -> float:
    p = counts[counts > 0] / n
    return float(-(p * np.log(p)).sum())


@dataclass
class QualityReport:
    nmi: float
    purity_a_to_b: float
    purity_b_to_a: float
    largest_jaccard: float
    communities_a: int
    communities_b: int
    largest_a: int
    largest_b: int


def compare_partitions(a: Sequence[int], b: Sequence[int]) -> QualityReport:
    """contingency_metrics (hit_leiden_incremental.rs:578-651) over the first
    min(len(a), len(b)) vertices."""
    a = np.asarray(a)
    b = np.asarray(b)
    n = min(len(a), len(b))
    if n == 0:
        return QualityReport(0.0, 0.0, 0.0, 0.0, 0, 0, 0, 0)
    a, b = a[:n], b[:n]
    ua, ia = np.unique(a, return_inverse=True)
    ub, ib = np.unique(b, return_inverse=True)
    ca = np.bincount(ia).astype(np.float64)
    cb = np.bincount(ib).astype(np.float64)
    pair = ia.astype(np.int64) * len(ub) + ib
    up, cp = np.unique(pair, return_counts=True)
    pa, pb = up // len(ub), up % len(ub)
    nf = float(n)
    ha, hb = _entropy(ca, nf), _entropy(cb, nf)
    p_hs = cp / nf
    mi = float((p_hs * np.log(p_hs / ((ca[pa] / nf) * (cb[pb] / nf)))).sum())
    nmi = mi / np.sqrt(ha * hb) if ha > 0.0 and hb > 0.0 else 0.0
    best_a = np.zeros(len(ua))
    np.maximum.at(best_a, pa, cp)
    best_b = np.zeros(len(ub))
    np.maximum.at(best_b, pb, cp)
    la, sa = largest_community(a)
    lb, sb = largest_community(b)
    ka = int(np.searchsorted(ua, la))
    kb = int(np.searchsorted(ub, lb))
    hit = np.nonzero((pa == ka) & (pb == kb))[0]
    inter = int(cp[hit[0]]) if len(hit) else 0
    union = sa + sb - inter
    jac = inter / union if union > 0 else 0.0
    return QualityReport(float(nmi), float(best_a.sum() / nf), float(best_b.sum() / nf),
                         float(jac), len(ua), len(ub), sa, sb)
