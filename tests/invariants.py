"""Quality invariants of a hierarchy, for GPU states and oracle states alike.

A state is given as per-level CSR (off, col, w) and maps f (community) and
s (sub-community = refined community) of that level's nodes.

* nested: s^p refines f^p, f^p = f^{p+1} ∘ s^p, and level p+1 has a node for
  every sub-community of level p;
* connected: every sub-community induces a connected subgraph of its level;
* local moves: no single node move gains more than `tol` modularity.

The reference's deterministic loops keep sub-communities connected; its
throughput refinement merges singletons Jacobi-style on a snapshot, so a
singleton can join a neighbour's sub-community while that neighbour leaves it
(throughput.rs:239-288), and about 15 % of the level-0 sub-communities come out
disconnected.  `disconnected_fraction` reports that number.
"""
import numpy as np


def _components(off, col, label):
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    n = len(off) - 1
    rows = np.repeat(np.arange(n), np.diff(off.astype(np.int64)))
    keep = label[rows] == label[col]
    a = sp.csr_matrix((np.ones(int(keep.sum())), (rows[keep], col[keep])), shape=(n, n))
    _, comp = connected_components(a, directed=False)
    return comp


def disconnected(off, col, s):
    """Number of sub-communities that are not connected, and of all of them."""
    comp = _components(off, col, s)
    pairs = np.unique(np.stack([s.astype(np.int64), comp.astype(np.int64)]), axis=1)
    ncls = len(np.unique(s))
    return pairs.shape[1] - ncls, ncls


def check_nested(levels):
    for p, (off, col, w, f, s) in enumerate(levels):
        pair = np.unique(np.stack([s.astype(np.int64), f.astype(np.int64)]), axis=1)
        assert len(np.unique(pair[0])) == pair.shape[1], f"level {p}: s does not refine f"
        if p + 1 < len(levels):
            f_up = levels[p + 1][3]
            assert len(f_up) >= len(np.unique(s)), f"level {p + 1} lacks nodes"
            assert np.array_equal(f, f_up[s]), f"level {p}: f != f^(p+1) o s"


def check_connected(levels):
    for p, (off, col, w, f, s) in enumerate(levels):
        bad, _ = disconnected(off, col, s)
        assert bad == 0, f"level {p}: {bad} sub-communities are not connected"


def max_move_gain(off, col, w, f, gamma=1.0):
    """Largest single-node move gain on a level (any-order sums: a bound, not
    parity)."""
    from oracle import oracle as O
    n = len(off) - 1
    rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off.astype(np.int64)))
    k = np.zeros(n)
    np.add.at(k, rows, w)
    tw = float(k.sum())
    if tw == 0.0:
        return 0.0
    d = np.zeros(int(max(int(f.max()) + 1, 2 * n + 2)))
    np.add.at(d, f, k)
    keep = rows < col
    loops = rows == col
    g = O.Graph.from_edges(n, np.concatenate([rows[keep], rows[loops][::2]]),
                           np.concatenate([col[keep], col[loops][::2]]),
                           np.concatenate([w[keep], w[loops][::2]]))
    _, gain = O.move_eval(g, f, d, k, tw, gamma, np.arange(n, dtype=np.uint32))
    return float(gain.max()) if n else 0.0


def check_local_moves(levels, tol=2e-3):
    for p, (off, col, w, f, s) in enumerate(levels):
        g = max_move_gain(off, col, w, f)
        assert g <= tol, (p, g)
