"""GPU stage-by-stage parity with the CPU oracle (bit-exact) and the reference
KATs replayed through the CUDA kernels.  Every call goes through libhl's C ABI.

Tolerance: bit-exact for every integer output and every FP64 value that feeds a
decision (weights, gains, community totals); modularity within 1e-12 relative.
"""
import importlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

gh = pytest.importorskip("tests.gpu_helpers")

SEEDS = list(range(6))


def _graph(seed, n=60, m=240, integral=True):
    rng = np.random.default_rng(seed)
    s, d, w = gh.random_graph(rng, n, m, integral)
    return rng, O.Graph.from_edges(n, s, d, w)


# ---- apply_delta (in_memory.rs:103-137) -----------------------------------
@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("keep_loops", [False, True])
def test_apply_delta_bit_exact(seed, integral, keep_loops):
    rng, g = _graph(seed, integral=integral)
    g = g.apply_delta([], [], [], keep_self_loops=True)  # canonical, duplicates merged
    off, col, w = g.csr()
    k = 80
    ds = rng.integers(0, g.n, k).astype(np.uint32)
    dd = rng.integers(0, g.n, k).astype(np.uint32)
    dw = rng.uniform(-2.5, 2.5, k) if not integral else rng.integers(-3, 4, k).astype(float)
    # exact deletes of existing edges and repeated keys
    for i in range(0, 20, 2):
        v = int(rng.integers(0, g.n))
        a, b = int(off[v]), int(off[v + 1])
        if b > a:
            j = int(rng.integers(a, b))
            ds[i], dd[i], dw[i] = v, col[j], -w[j]
    ds[30:34] = ds[29]
    dd[30:34] = dd[29]
    ds[40], dd[40] = 5, 5  # a self-loop in the delta
    dw[40] = 3.0
    ref = g.apply_delta(ds, dd, dw, keep_self_loops=keep_loops)
    go, gc, gw = gh.apply_delta(g, ds, dd, dw, keep_loops)
    ro, rc, rw = ref.csr()
    assert gh.same_bits(go, ro) and gh.same_bits(gc, rc) and gh.same_bits(gw, rw)


@pytest.mark.parametrize("before", [30, 31, 32, 63])
@pytest.mark.parametrize("keep_loops", [False, True])
def test_apply_delta_self_loop_across_chunks(before, keep_loops):
    # The self-loop of vertex v is stored twice in its row, at positions
    # `before` and `before + 1`: the warp merge reads rows 32 entries at a time,
    # so the two copies sit in one chunk or straddle two.
    n = 200
    v = 150
    nb = list(range(before)) + list(range(v + 1, v + 11))
    src = [v] * len(nb) + [v]
    dst = nb + [v]
    w = [1.0 + 0.25 * (i % 5) for i in range(len(nb))] + [4.0]
    g = O.Graph.from_edges(n, src, dst, w).apply_delta([], [], [], keep_self_loops=True)
    off, col, _ = g.csr()
    row = col[off[v]:off[v + 1]].tolist()
    assert row[before] == v and row[before + 1] == v
    cases = [([v], [v], [-4.0]),                        # delete the loop
             ([v, v, 3], [v, v + 20, 4], [-4.0, 2.0, 1.0]),  # delete it, insert around it
             ([v, 0], [v, v], [1.5, -1.0]),             # reweight it, delete an edge before it
             ([v, 7], [v + 30, 8], [1.0, 1.0])]         # untouched loop in a touched row
    for ds, dd, dw in cases:
        ref = g.apply_delta(ds, dd, dw, keep_self_loops=keep_loops)
        go, gc, gw = gh.apply_delta(g, ds, dd, dw, keep_loops)
        ro, rc, rw = ref.csr()
        assert gh.same_bits(go, ro) and gh.same_bits(gc, rc) and gh.same_bits(gw, rw)


@pytest.mark.parametrize("total,before", [(5120, 2558), (5120, 2559), (5120, 2560),
                                          (600, 222), (600, 223), (600, 224)])
@pytest.mark.parametrize("keep_loops", [False, True])
def test_apply_delta_long_rows_split_across_warps(total, before, keep_loops):
    # A row above 512 entries is merged by a whole block, its 8 warps on
    # consecutive slices of 32-entry chunks.  With 5120 neighbours and a
    # self-loop the row has 161 chunks and a slice starts at entry 2560; with
    # 600 it has 19 chunks and a slice starts at entry 224.  The loop's two
    # copies sit just before, across, or just after that boundary.
    rng = np.random.default_rng(before)
    n = 9000
    v = 4000
    nb = list(range(before)) + list(range(v + 1, v + 1 + total - before))
    src = [v] * len(nb) + [v]
    dst = nb + [v]
    w = list(rng.uniform(0.5, 2.0, len(nb))) + [3.0]
    g = O.Graph.from_edges(n, src, dst, w).apply_delta([], [], [], keep_self_loops=True)
    off, col, ww = g.csr()
    row = col[off[v]:off[v + 1]]
    assert row[before] == v and row[before + 1] == v
    # deletes of existing row entries, inserts of new neighbours on both sides
    # of the loop, the loop itself deleted or reweighted
    k = min(400, total // 4)
    dels = rng.choice(len(nb), k, replace=False)
    new_nb = rng.choice(np.setdiff1d(np.arange(n), np.array(nb + [v])), k, replace=False)
    for loop_w in (-3.0, 1.25):
        ds = [v] * (len(dels) + len(new_nb)) + [v]
        dd = [nb[i] for i in dels] + new_nb.tolist() + [v]
        dw = [-w[i] for i in dels] + rng.uniform(0.5, 2.0, len(new_nb)).tolist() + [loop_w]
        ref = g.apply_delta(ds, dd, dw, keep_self_loops=keep_loops)
        go, gc, gw = gh.apply_delta(g, ds, dd, dw, keep_loops)
        ro, rc, rw = ref.csr()
        assert gh.same_bits(go, ro) and gh.same_bits(gc, rc) and gh.same_bits(gw, rw)


def test_apply_delta_drops_existing_self_loops():
    g = O.Graph.from_edges(3, [0, 0], [0, 1], [5.0, 1.0])
    off, col, w = gh.apply_delta(g, [2], [2], [3.0], keep_loops=False)
    assert col.tolist() == [1, 0, 2, 2] and w.tolist() == [1.0, 1.0, 3.0, 3.0]


def test_apply_delta_kats():
    g = O.Graph.from_edges(4, [0, 1, 0], [1, 2, 2], [1.0, 1.0, 1.0])
    off, col, w = gh.apply_delta(g, [2], [3], [1.0])
    assert 2 in col[off[3]:off[4]].tolist() and 3 in col[off[2]:off[3]].tolist()
    assert abs(w.sum() / 2 - 4.0) < 1e-9
    g3 = O.Graph.from_edges(3, [0, 1, 0], [1, 2, 2], [1.0, 1.0, 1.0])
    off, col, w = gh.apply_delta(g3, [0], [2], [-1.0])
    assert col[off[0]:off[1]].tolist() == [1]


# ---- per-vertex decisions on a fixed snapshot (parallel_frontier.rs:133-239)
@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("integral", [True, False])
def test_move_eval_bit_exact(seed, integral):
    rng, g = _graph(seed, n=300, m=3000, integral=integral)
    # hubs so that the shared-memory and global hash paths are exercised
    hub_src = np.repeat(np.arange(3, dtype=np.uint32), 400)
    hub_dst = rng.integers(3, 300, len(hub_src)).astype(np.uint32)
    src, dst, w = gh.random_graph(rng, 300, 3000, integral)
    src = np.concatenate([src, hub_src])
    dst = np.concatenate([dst, hub_dst])
    w = np.concatenate([w, rng.integers(1, 3, len(hub_src)).astype(float) if integral
                        else rng.uniform(0.5, 2, len(hub_src))])
    g = O.Graph.from_edges(300, src, dst, w).apply_delta([], [], [], keep_self_loops=True)
    n = g.n
    for k_comm in [3, 20, 150]:
        f = gh.random_partition(rng, n, k_comm)
        k = g.degrees()
        tw = O.tree_sum(k)
        d = np.zeros(2 * n + 2)
        np.add.at(d, f, k)
        verts = np.arange(n, dtype=np.uint32)
        for gamma in [0.5, 1.0, 3.0]:
            to_o, g_o = O.move_eval(g, f, d, k, tw, gamma, verts)
            to_g, g_g = gh.move_eval(g, f, d, k, tw, gamma, verts)
            assert gh.same_bits(g_o, g_g)
            pos = g_o > 0
            assert np.array_equal(to_o[pos], to_g[pos])


# ---- decoupled selection (throughput.rs:204-236) -------------------------
def test_select_kats():
    assert gh.select_decoupled([1, 2, 3], [10, 20, 30], [20, 10, 40], [10.0, 9.0, 8.0]).tolist() == [1, 3]
    assert gh.select_decoupled([10, 11, 12, 13], [1, 1, 4, 2], [2, 3, 2, 5],
                               [10.0, 9.0, 8.0, 7.0]).tolist() == [10, 11, 12]
    assert gh.select_decoupled([7, 3], [1, 2], [2, 1], [5.0, 5.0]).tolist() == [3]


@pytest.mark.parametrize("seed", list(range(10)))
@pytest.mark.parametrize("ncomm", [4, 30, 3000])
def test_select_random_matches_greedy(seed, ncomm):
    rng = np.random.default_rng(100 + seed)
    m = 5000
    node = rng.permutation(m).astype(np.uint32)
    frm = rng.integers(0, ncomm, m).astype(np.uint32)
    to = rng.integers(0, ncomm, m).astype(np.uint32)
    gain = rng.integers(1, 50, m).astype(float)  # many exact ties
    ref = O.select_decoupled(node, frm, to, gain)
    got = gh.select_decoupled(node, frm, to, gain)
    assert np.array_equal(ref, got)


# ---- inc_movement (hit_leiden.rs:1024-1101) --------------------------------
@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("mark", [False, True])
def test_inc_movement_bit_exact(seed, integral, mark):
    rng, g = _graph(seed, n=400, m=2500, integral=integral)
    g = g.apply_delta([], [], [], keep_self_loops=True)
    n = g.n
    f0 = gh.random_partition(rng, n, 40)
    s = gh.random_partition(rng, n, 120)
    ds = rng.integers(0, n, 30).astype(np.uint32)
    dd = rng.integers(0, n, 30).astype(np.uint32)
    dw = rng.choice([-1.0, 1.0, 2.0], 30)
    for delta in [([], [], []), (ds, dd, dw)]:
        fo, cho, afo, ito = O.inc_movement(g, *delta, f0, s, 1.0, O.MODE_THROUGHPUT,
                                           mark_moved=mark)
        fg, chg, afg, itg = gh.inc_movement(g, *delta, f0, s, 1.0, mark_moved=mark)
        assert np.array_equal(fo, fg)
        assert np.array_equal(cho, chg)
        assert np.array_equal(afo, afg)
        assert ito == itg


def test_inc_movement_compacts_ids_at_or_above_n():
    g = O.Graph.from_edges(4, [0, 1, 2], [1, 2, 3], [1.0, 1.0, 1.0])
    f0 = [7, 7, 9, 9]  # ids >= n: ranked to 0, 0, 1, 1 first
    fo, *_ = O.inc_movement(g, [], [], [], f0, [0, 1, 2, 3], 1.0, O.MODE_THROUGHPUT)
    fg, *_ = gh.inc_movement(g, [], [], [], f0, [0, 1, 2, 3], 1.0)
    assert np.array_equal(fo, fg)


# ---- reference KATs for movement through the GPU ------------------------------
def test_gpu_kat_empty_community():
    g = O.Graph.from_edges(3, [0, 0], [1, 2], [10.0, 0.5])
    f, *_ = gh.inc_movement(g, [], [], [], [0, 0, 0], [0, 0, 0], 3.0)
    assert f[2] != f[0]


def test_gpu_kat_no_move_k4():
    g = O.Graph.from_edges(4, [0, 0, 0, 1, 1, 2], [1, 2, 3, 2, 3, 3])
    f, ch, *_ = gh.inc_movement(g, [], [], [], [0] * 4, [0, 1, 2, 3], 1.0)
    assert not ch.any()


def test_gpu_kat_intra_deletion_activates():
    g = O.Graph.from_edges(4, [0, 2], [1, 3], [10.0, 10.0])
    f, ch, *_ = gh.inc_movement(g, [0], [2], [-1.0], [0, 0, 0, 1], [0, 1, 2, 3], 1.0)
    assert f[2] == f[3] and ch[2]


# ---- inc_refinement (hit_leiden.rs:1265-1390) ---------------------------------
@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("same_f", [False, True])
@pytest.mark.parametrize("exact", [False, True])
def test_inc_refinement_bit_exact(seed, integral, same_f, exact):
    rng, g = _graph(seed, n=400, m=1200, integral=integral)
    g = g.apply_delta([], [], [], keep_self_loops=True)
    n = g.n
    f = gh.random_partition(rng, n, 10)
    for s0 in [np.arange(n, dtype=np.uint32), gh.random_partition(rng, n, 30),
               (f * 3 + rng.integers(0, 3, n)).astype(np.uint32)]:
        aff = rng.random(n) < 0.3
        so = s0.copy()
        ref_s, ref_r = _oracle_refine(g, f, so, aff, same_f)
        with gh.exact_tfilter(exact):
            gs, gr = gh.inc_refinement(g, f, s0, aff, 1.0, same_f)
        assert np.array_equal(ref_s, gs)
        assert np.array_equal(ref_r, gr)


def _oracle_refine(g, f, s, aff, same_f):
    return O.inc_refinement(g, f, s, aff, 1.0, O.MODE_THROUGHPUT, cc_same_community=same_f)


def test_gpu_kat_refinement():
    g = O.Graph.from_edges(4, [0, 0, 1, 1], [1, 3, 3, 2], [10.0, 100.0, 100.0, 1.0])
    s, r = gh.inc_refinement(g, [0, 0, 0, 1], [0, 1, 2, 3], [1, 1, 1, 1], 1.0)
    assert s[2] == 2  # T-filter (hit_leiden.rs:2058-2114)
    g = O.Graph.from_edges(5, [0, 1, 3], [1, 2, 4])
    s, r = gh.inc_refinement(g, [0] * 5, [0] * 5, [1] * 5, 1.0)
    assert s[:3].tolist() == [0, 0, 0] and s[3] != 0 and s[3] == s[4]
    g = O.Graph.from_edges(4, [0, 2], [1, 3])
    s, r = gh.inc_refinement(g, [0] * 4, [0] * 4, [1] * 4, 1.0)
    assert s.tolist() == [1, 1, 0, 0]  # equal components: the last keeps the id
    s, r = gh.inc_refinement(g, [0, 0, 1, 1], [0, 0, 2, 2], [0, 0, 1, 1], 1.0)
    assert s[0] == 0 and s[1] == 0


# ---- inc_aggregation (hit_leiden.rs:1639-1731) --------------------------------
@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("flags", [0, O.FLAG_AGG_CHANGED_ONLY | O.FLAG_EDGE_WEIGHT_LOOPS])
def test_inc_aggregation_bit_exact(seed, integral, flags):
    rng = np.random.default_rng(seed)
    n = 300
    src, dst, w = gh.random_graph(rng, n, 1500, integral, loops=0.1)
    g = O.Graph.from_edges(n, src, dst, w).apply_delta([], [], [], keep_self_loops=True)
    s_pre = gh.random_partition(rng, n, 80)
    s_cur = s_pre.copy()
    moved = rng.random(n) < 0.2
    s_cur[moved] = rng.integers(0, 120, moved.sum())
    refined = moved | (rng.random(n) < 0.05)
    ds = rng.integers(0, n, 50).astype(np.uint32)
    dd = rng.integers(0, n, 50).astype(np.uint32)
    dw = rng.choice([-1.0, 1.0, 0.5], 50)
    (ou, ov, ow), nsp, nn = O.inc_aggregation(g, ds, dd, dw, s_pre, s_cur, refined, flags)
    co = bool(flags & O.FLAG_AGG_CHANGED_ONLY)
    ew = bool(flags & O.FLAG_EDGE_WEIGHT_LOOPS)
    (gu, gv, gw), gsp, gn = gh.inc_aggregation(g, ds, dd, dw, s_pre, s_cur, refined, co, ew)
    assert np.array_equal(ou, gu) and np.array_equal(ov, gv) and gh.same_bits(ow, gw)
    assert np.array_equal(nsp, gsp) and nn == gn


def test_gpu_kat_aggregation():
    g = O.Graph.from_edges(4, [0, 1, 2], [1, 2, 3])
    (u, v, w), _, _ = gh.inc_aggregation(g, [0], [2], [5.0], [0, 0, 2, 2], [0, 0, 0, 2], [0] * 4)
    assert list(zip(u.tolist(), v.tolist(), w.tolist())) == [(0, 2, 5.0)]
    g = O.Graph.from_edges(4, [0, 2], [1, 3])
    (u, v, w), _, _ = gh.inc_aggregation(g, [0, 0], [2, 3], [3.0, -3.0], [0, 0, 1, 1],
                                         [0, 0, 1, 1], [0] * 4)
    assert len(u) == 0
    g = O.Graph.from_edges(3, [0, 0, 1], [0, 1, 2], [5.0, 1.0, 1.0])
    (u, v, w), _, _ = gh.inc_aggregation(g, [], [], [], [0, 1, 2], [1, 1, 2], [1, 0, 0])
    sl = {(a, b): x for a, b, x in zip(u.tolist(), v.tolist(), w.tolist())}
    assert sl[(0, 0)] == -10.0 and sl[(1, 1)] > 0


# ---- 2m and modularity ----------------------------------------------------------
@pytest.mark.parametrize("n", [1, 7, 1024, 1025, 70000, 2 ** 20 + 3])
def test_tree_sum_bit_exact(n):
    x = np.random.default_rng(n).uniform(0.1, 3.0, n)
    assert gh.same_bits(np.array([O.tree_sum(x)]), np.array([gh.tree_sum(x)]))


@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("integral", [True, False])
def test_modularity_close(seed, integral):
    rng, g = _graph(seed, n=500, m=4000, integral=integral)
    for k in [1, 7, 60, 500]:
        part = gh.random_partition(rng, g.n, k)
        qo = O.modularity_csr(g, part)
        qg = gh.modularity(g, part)
        assert abs(qo - qg) <= 1e-12 * max(1.0, abs(qo))


def test_modularity_kats():
    tri = O.Graph.from_edges(3, [0, 1, 0], [1, 2, 2])
    assert abs(gh.modularity(tri, [0, 0, 0])) < 1e-12
    assert abs(gh.modularity(tri, [0, 1, 2]) + 1.0 / 3.0) < 1e-12
    two = O.Graph.from_edges(6, [0, 1, 0, 3, 4, 3], [1, 2, 2, 4, 5, 5])
    assert abs(gh.modularity(two, [0, 0, 0, 1, 1, 1]) - 0.5) < 1e-12
    e = O.Graph.from_edges(3, [], [])
    assert gh.modularity(e, [0, 1, 2]) == 0.0
    p = O.Graph.from_edges(2, [0], [1], [5.0])
    assert abs(gh.modularity(p, [0, 0])) < 1e-12 and abs(gh.modularity(p, [0, 1]) + 0.5) < 1e-12


def test_canonicalize_gpu():
    hl = gh.hl
    assert hl.canonicalize_community_ids([5, 5, 3, 3, 7]).tolist() == [0, 0, 1, 1, 2]
    x = np.random.default_rng(1).integers(0, 1000, 100000)
    assert np.array_equal(hl.canonicalize_community_ids(x), O.canonicalize(x))


# ---- integral hub rows through either hub path: the block kernel's shared
# tables (no direct deferral) or the partitioned pass (every hub row) -------
@pytest.mark.parametrize("defer", [1, 0xFFFFFFFF, 0])
def test_move_eval_hub_paths_bit_exact(defer):
    rng = np.random.default_rng(defer & 0xFFFF)
    n = 60000
    src, dst, w = gh.random_graph(rng, n, 40000, True)
    hubs = [(0, 700), (1, 3000), (2, 9000), (3, 40000)]
    hs, hd = [], []
    for h, deg in hubs:
        nb = rng.choice(np.arange(10, n), deg, replace=False).astype(np.uint32)
        hs.append(np.full(deg, h, np.uint32))
        hd.append(nb)
    hw = rng.integers(1, 4, sum(d for _, d in hubs)).astype(float)
    g = O.Graph.from_edges(n, np.concatenate([src] + hs), np.concatenate([dst] + hd),
                           np.concatenate([w, hw])).apply_delta([], [], [], keep_self_loops=True)
    k = g.degrees()
    tw = O.tree_sum(k)
    for ncomm in [7, 3000, 50000]:
        f = gh.random_partition(rng, n, ncomm)
        # a heavy key: 30 % of the largest hub's neighbours in one community
        heavy = hd[-1][: len(hd[-1]) * 3 // 10]
        f[heavy] = f[hd[-1][0]]
        d = np.zeros(2 * n + 2)
        np.add.at(d, f, k)
        verts = np.concatenate([np.arange(4, dtype=np.uint32),
                                np.arange(4, n, 11, dtype=np.uint32)])
        to_o, g_o = O.move_eval(g, f, d, k, tw, 1.0, verts)
        with gh.hub_defer(defer):
            to_g, g_g = gh.move_eval(g, f, d, k, tw, 1.0, verts)
        assert gh.same_bits(g_o, g_g)
        pos = g_o > 0
        assert np.array_equal(to_o[pos], to_g[pos])


# ---- integral weights too large for a 32-bit group sum (>= 2^26 each): the
# lanes that share a key are added up by their leader instead -----------------
@pytest.mark.parametrize("defer", [1, 0xFFFFFFFF])
def test_move_eval_hub_large_integral_weights(defer):
    rng = np.random.default_rng(7 + (defer & 3))
    n = 30000
    src, dst, w = gh.random_graph(rng, n, 20000, True)
    w = w * float(1 << 27)
    hubs = [(0, 1500), (1, 12000)]
    hs, hd = [], []
    for h, deg in hubs:
        hs.append(np.full(deg, h, np.uint32))
        hd.append(rng.choice(np.arange(10, n), deg, replace=False).astype(np.uint32))
    hw = rng.integers(1 << 27, 1 << 30, sum(d for _, d in hubs)).astype(float)
    g = O.Graph.from_edges(n, np.concatenate([src] + hs), np.concatenate([dst] + hd),
                           np.concatenate([w, hw])).apply_delta([], [], [], keep_self_loops=True)
    k = g.degrees()
    tw = O.tree_sum(k)
    assert tw < 2.0 ** 52  # integral sums stay exact
    for ncomm in [5, 2000]:
        f = gh.random_partition(rng, n, ncomm)
        heavy = hd[-1][: len(hd[-1]) // 2]  # half of the big hub's row in one key
        f[heavy] = f[hd[-1][0]]
        d = np.zeros(2 * n + 2)
        np.add.at(d, f, k)
        verts = np.concatenate([np.arange(2, dtype=np.uint32),
                                np.arange(2, n, 13, dtype=np.uint32)])
        to_o, g_o = O.move_eval(g, f, d, k, tw, 1.0, verts)
        with gh.hub_defer(defer):
            to_g, g_g = gh.move_eval(g, f, d, k, tw, 1.0, verts)
        assert gh.same_bits(g_o, g_g)
        pos = g_o > 0
        assert np.array_equal(to_o[pos], to_g[pos])


# ---- very high degree vertices (block kernel, shared and global tables) -----
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("hub_deg", [300, 3000, 6000, 20000])
@pytest.mark.parametrize("slots", [0, 64])
def test_move_eval_hubs_bit_exact(integral, hub_deg, slots):
    rng = np.random.default_rng(hub_deg)
    n = max(9000, hub_deg + 1000)
    src, dst, w = gh.random_graph(rng, n, 20000, integral)
    hs = np.zeros(hub_deg, np.uint32)
    hd = rng.choice(np.arange(1, n), hub_deg, replace=False).astype(np.uint32)
    hw = rng.integers(1, 3, hub_deg).astype(float) if integral else rng.uniform(0.5, 2, hub_deg)
    g = O.Graph.from_edges(n, np.concatenate([src, hs]), np.concatenate([dst, hd]),
                           np.concatenate([w, hw])).apply_delta([], [], [], keep_self_loops=True)
    k = g.degrees()
    tw = O.tree_sum(k)
    for ncomm in [5, 400, 4000]:
        f = gh.random_partition(rng, n, ncomm)
        d = np.zeros(2 * n + 2)
        np.add.at(d, f, k)
        verts = np.arange(0, n, 7, dtype=np.uint32)
        to_o, g_o = O.move_eval(g, f, d, k, tw, 1.0, verts)
        with gh.bucket_slots(slots):  # 64: buckets overflow, rows take the global tables
            to_g, g_g = gh.move_eval(g, f, d, k, tw, 1.0, verts)
        assert gh.same_bits(g_o, g_g)
        pos = g_o > 0
        assert np.array_equal(to_o[pos], to_g[pos])


@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("ncomm", [1, 3])
@pytest.mark.parametrize("exact", [False, True])
def test_inc_refinement_hub_bit_exact(integral, ncomm, exact):
    rng = np.random.default_rng(7)
    n = 7000
    src, dst, w = gh.random_graph(rng, n, 15000, integral)
    hd = rng.choice(np.arange(1, n), 5000, replace=False).astype(np.uint32)
    hw = np.ones(5000) if integral else rng.uniform(0.5, 2, 5000)
    g = O.Graph.from_edges(n, np.concatenate([src, np.zeros(5000, np.uint32)]),
                           np.concatenate([dst, hd]), np.concatenate([w, hw])
                           ).apply_delta([], [], [], keep_self_loops=True)
    # one community: the hub sees ~5000 distinct sub-communities (global table)
    f = gh.random_partition(rng, n, ncomm)
    s0 = np.arange(n, dtype=np.uint32)
    aff = np.ones(n, bool)
    ref_s, ref_r = O.inc_refinement(g, f, s0, aff, 1.0, O.MODE_THROUGHPUT)
    with gh.exact_tfilter(exact):
        gs, gr = gh.inc_refinement(g, f, s0, aff, 1.0)
    assert np.array_equal(ref_s, gs) and np.array_equal(ref_r, gr)


# ---- degree-bin thresholds (the autotuner's candidates) -------------------
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("pair", [(128, 512), (64, 512), (128, 256), (64, 256), (96, 384),
                                  (33, 33)])
def test_move_eval_same_for_every_bin_split(integral, pair):
    rng = np.random.default_rng(31)
    n = 12000
    src, dst, w = gh.random_graph(rng, n, 60000, integral)
    # a spread of degrees across every bin: a few vertices of 40..1500 entries
    hubs = rng.choice(n, 40, replace=False).astype(np.uint32)
    hs, hd = [], []
    for i, h in enumerate(hubs):
        deg = int(40 + 40 * i)
        hs.append(np.full(deg, h, np.uint32))
        hd.append(rng.choice(n, deg, replace=False).astype(np.uint32))
    hs, hd = np.concatenate(hs), np.concatenate(hd)
    keep = hs != hd
    hw = (rng.integers(1, 3, keep.sum()).astype(float) if integral
          else rng.uniform(0.5, 2, keep.sum()))
    g = O.Graph.from_edges(n, np.concatenate([src, hs[keep]]), np.concatenate([dst, hd[keep]]),
                           np.concatenate([w, hw])).apply_delta([], [], [], keep_self_loops=True)
    k = g.degrees()
    tw = O.tree_sum(k)
    f = gh.random_partition(rng, n, 300)
    d = np.zeros(2 * n + 2)
    np.add.at(d, f, k)
    verts = np.arange(n, dtype=np.uint32)
    to_o, g_o = O.move_eval(g, f, d, k, tw, 1.0, verts)
    with gh.bins(*pair):
        to_g, g_g = gh.move_eval(g, f, d, k, tw, 1.0, verts)
    assert gh.same_bits(g_o, g_g)
    pos = g_o > 0
    assert np.array_equal(to_o[pos], to_g[pos])


def test_autotuned_handle_stays_bit_exact():
    """A frontier of at least 20,000 vertices triggers the degree-bin
    autotuner; the state stays bit-exact with the oracle through it."""
    import ctypes as C
    hl = importlib.import_module("hit-leiden_b200")
    L = importlib.import_module("hit-leiden_b200._lib")
    E2E = importlib.import_module("tests.test_gpu_e2e")
    W = importlib.import_module("hit-leiden_b200.workloads")
    n, s, d, w = W.config2(4, n=40_000, mean_degree=12.0)
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("t", n, s, d, w),
                                hl.RunConfig(mode=hl.RunMode.Throughput))
    os_ = E2E.oracle_state(n, s, d, w, 10)
    gs.apply_batch([], [], [])  # empty batch: every vertex active at level 0
    os_.hit_leiden([], [], [])
    mid, wide, hd, fr = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    L.check(L.lib.hl_autotune_info(gs._h, C.byref(mid), C.byref(wide), C.byref(hd),
                                   C.byref(fr)))
    assert fr.value >= 20000 and 33 <= mid.value <= 128 and mid.value <= wide.value <= 512
    assert hd.value in (1, 2048, 8192, 32768)
    E2E.compare(gs, os_)
    store = W.EdgeStore(n, s, d, w)
    u, v, ww = W.mixed_batch(store, 500, 0.9, 8, weights=(0.5, 2.0), preferential=True)
    gs.apply_batch(u, v, ww)
    os_.hit_leiden(u, v, ww)
    E2E.compare(gs, os_)
    gs.close()
