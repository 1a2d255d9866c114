"""Structural invariants of the oracle's multi-level state after a bootstrap and
after incremental batches (the checker the GPU state is compared against bit
for bit).

At every level p below the top:
- every level holds the same total weight (aggregation conserves it);
- the maps agree top-down: f_p(v) = f_{p+1}(s_p(v)) (def_update,
  hit_leiden.rs:1766-1793);
- s_p maps into the nodes of level p+1;
- level p+1's supergraph is level p's CSR aggregated by s_p, computed here from
  scratch: the incremental ΔH path (hit_leiden.rs:1639-1731) and a static
  aggregation must give the same graph.  A super-node's self-loop is stored
  twice, and its two copies sum to the weight of the entries inside it.
And level 0's modularity equals a recomputation from its CSR.

Integral weights make every sum exact; with f64 weights the comparison allows
1e-9 relative (the oracle sums in push order, numpy in its own)."""
import importlib

import numpy as np
import pytest

from oracle import oracle as O

W = importlib.import_module("hit-leiden_b200.workloads")


def _aggregate(off, col, w, s, n_next):
    rows = np.repeat(np.arange(len(off) - 1), np.diff(off).astype(np.int64))
    keys = s[rows].astype(np.int64) * n_next + s[col].astype(np.int64)
    uk, inv = np.unique(keys, return_inverse=True)
    return uk, np.bincount(inv, weights=w, minlength=len(uk))


def _entries(off, col, w, n):
    rows = np.repeat(np.arange(len(off) - 1), np.diff(off).astype(np.int64))
    keys = rows.astype(np.int64) * n + col.astype(np.int64)
    uk, inv = np.unique(keys, return_inverse=True)
    return uk, np.bincount(inv, weights=w, minlength=len(uk))


def _check(st, rel):
    P = st.levels
    tw0 = st.graph(0).total_weight()
    for p in range(P):
        assert st.graph(p).total_weight() == pytest.approx(tw0, rel=rel, abs=0), p
    for p in range(P - 1):
        g, g1 = st.graph(p), st.graph(p + 1)
        f = st.get_map(p, O.MAP_F)
        s = st.get_map(p, O.MAP_S_CUR)
        f1 = st.get_map(p + 1, O.MAP_F)
        assert len(s) == g.n and (len(s) == 0 or int(s.max()) < g1.n), p
        assert np.array_equal(f, f1[s]), p
        off, col, w = g.csr()
        k_want, w_want = _aggregate(off, col, w, s, g1.n)
        o1, c1, ww1 = g1.csr()
        k_got, w_got = _entries(o1, c1, ww1, g1.n)
        assert np.array_equal(k_want, k_got), p
        np.testing.assert_allclose(w_got, w_want, rtol=rel, atol=0)
    off, col, w = st.graph(0).csr()
    rows = np.repeat(np.arange(len(off) - 1), np.diff(off).astype(np.int64)).astype(np.uint32)
    # each undirected edge once (a self-loop's two stored copies as one edge)
    keep = rows < col
    loops = rows == col
    src = np.concatenate([rows[keep], rows[loops][::2]])
    dst = np.concatenate([col[keep], col[loops][::2]])
    ww = np.concatenate([w[keep], w[loops][::2]])
    q = O.modularity_edges(st.graph(0).n, src, dst, ww, st.get_map(0, O.MAP_F))
    assert q == pytest.approx(st.modularity(0), rel=1e-9, abs=1e-12)


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("weights", [None, (0.5, 2.0)])
def test_invariants_after_bootstrap_and_batches(seed, weights):
    rel = 0 if weights is None else 1e-9
    n, s, d, w, _ = W.planted(1500, 8.0, 0.25, seed, comm_min=5, comm_max=80, weights=weights)
    st = O.State(n, mode=O.MODE_THROUGHPUT)
    st.bootstrap(s, d, w, max_levels=10)
    _check(st, rel)
    store = W.EdgeStore(n, s, d, w)
    for b in range(3):
        u, v, ww = W.mixed_batch(store, 150, 0.8, 100 * seed + b, weights=weights,
                                 preferential=False)
        st.hit_leiden(u, v, ww)
        _check(st, rel)


@pytest.mark.parametrize("seed", [3, 4])
def test_invariants_under_delete_heavy_batches(seed):
    # 70 % deletes: communities shrink and split rather than grow
    n, s, d, w, _ = W.planted(1500, 10.0, 0.2, seed, comm_min=5, comm_max=80)
    st = O.State(n, mode=O.MODE_THROUGHPUT)
    st.bootstrap(s, d, w, max_levels=10)
    store = W.EdgeStore(n, s, d, w)
    for b in range(5):
        u, v, ww = W.mixed_batch(store, 300, 0.3, 50 * seed + b, preferential=False)
        st.hit_leiden(u, v, ww)
        _check(st, 0)


def _levels_of(st):
    out = []
    for p in range(st.levels):
        off, col, w = st.graph(p).csr()
        out.append((off, col, w, st.get_map(p, O.MAP_F), st.get_map(p, O.MAP_S_CUR)))
    return out


@pytest.mark.parametrize("mode", [O.MODE_DETERMINISTIC, O.MODE_THROUGHPUT])
@pytest.mark.parametrize("seed", [0, 1])
def test_hierarchy_quality_invariants(mode, seed):
    """Nesting and local optimality (no single move gains more than 2e-3) in
    both modes; connected sub-communities at every level in deterministic
    mode (the nodes a level gains from splits below join K there, M8)."""
    import importlib
    INV = importlib.import_module("tests.invariants")
    n, s, d, w = W.config1(seed)
    st = O.State(n, mode=mode)
    st.bootstrap(s, d, w, max_levels=10)
    ex = set(zip(s.tolist(), d.tolist()))
    for b in range(4):
        u, v, ww = W.uniform_inserts(n, 1000, 7000 + 10 * seed + b, ex)
        st.hit_leiden(u, v, ww)
    lv = _levels_of(st)
    INV.check_nested(lv)
    INV.check_local_moves(lv)
    if mode == O.MODE_DETERMINISTIC:
        INV.check_connected(lv)
    else:
        bad, total = INV.disconnected(*lv[0][:2], lv[0][4])
        assert 0 < bad < 0.25 * total  # the Jacobi merges' known effect
