"""The throughput best-move evaluation (parallel_frontier.rs:150-230), the
decoupled move selection (throughput.rs:204-236), the throughput movement
loop around them (hit_leiden.rs:1024-1101, throughput.rs:80-202), the
throughput refinement (hit_leiden.rs:1265-1390, 1554-1637,
throughput.rs:239-359), apply_delta (in_memory.rs:103-137) and
inc_aggregation (hit_leiden.rs:1639-1731) restated a second time, in plain
Python straight from the reference, and compared bit for bit with the oracle
on random inputs; and modularity (hit_leiden.rs:121-161) evaluated exactly in
rationals, which the oracle must meet within 1e-12 relative.  The GPU's evaluation
kernels are compared with the oracle in test_gpu_parity.py, so this pins the
two restatements to each other.

Python floats are IEEE doubles and every expression keeps the reference's
operation order, so equality is exact: neighbour weights summed per community
in CSR order, candidates in first-encounter order, strict `>` from a best
gain of 0.0, and the empty community n + v last."""
import numpy as np
import pytest

from oracle import oracle as O


def best_move(off, col, w, v, f, d, k, tw, gamma, n):
    cur = int(f[v])
    kv = float(k[v])
    best, bestg = cur, 0.0
    wcur = 0.0
    buf, dirty = {}, []
    for p in range(int(off[v]), int(off[v + 1])):
        nb = int(col[p])
        if nb == v:
            continue  # self-loops are skipped
        c = int(f[nb])
        if buf.get(c, 0.0) == 0.0:
            dirty.append(c)
        buf[c] = buf.get(c, 0.0) + float(w[p])
        if c == cur:
            wcur += float(w[p])
    dcur = float(d[cur])
    for c in dirty:
        if c == cur:
            continue
        g = (buf[c] - wcur) / tw + gamma * kv * (dcur - kv - float(d[c])) / (tw * tw)
        if g > bestg:
            best, bestg = c, g
    eg = -wcur / tw + gamma * kv * (dcur - kv) / (tw * tw)
    if eg > bestg:
        best, bestg = n + v, eg
    return best, bestg


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("gamma", [0.5, 1.0, 3.0])
def test_move_eval_matches_restatement(seed, integral, gamma):
    rng = np.random.default_rng(seed)
    n, m = 300, 1500
    s = rng.integers(0, n, m)
    t = rng.integers(0, n, m)
    s[:10] = t[:10]  # a few self-loops
    w = rng.integers(1, 4, m).astype(float) if integral else rng.uniform(0.5, 2.0, m)
    g = O.Graph.from_edges(n, s.astype(np.uint32), t.astype(np.uint32), w)
    off, col, ww = g.csr()
    k = g.degrees()
    tw = g.total_weight() * 2.0
    f = rng.integers(0, 25, n).astype(np.uint32)
    d = np.zeros(2 * n + 2)
    for v in range(n):
        d[f[v]] += k[v]
    verts = np.arange(n, dtype=np.uint32)
    to, gain = O.move_eval(g, f, d, k, tw, gamma, verts)
    moves = 0
    for v in range(n):
        bt, bg = best_move(off, col, ww, v, f, d, k, tw, gamma, n)
        assert (int(to[v]), np.float64(gain[v]).view(np.uint64)) == \
            (bt, np.float64(bg).view(np.uint64)), v
        moves += bt != f[v]
    assert moves > 0


def select_moves(node, frm, to, gain):
    """throughput.rs:204-236: sort by gain descending then node ascending
    (stable), then accept a move iff its gain is positive, its node has not
    moved, it leaves no acceptor and enters no emitter."""
    order = sorted(range(len(node)), key=lambda i: (-float(gain[i]), int(node[i])))
    emitters, acceptors, moved, out = set(), set(), set(), []
    for i in order:
        if gain[i] <= 0.0 or node[i] in moved:
            continue
        if frm[i] in acceptors or to[i] in emitters:
            continue
        out.append(int(node[i]))
        moved.add(node[i])
        emitters.add(frm[i])
        acceptors.add(to[i])
    return out


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("ncomm", [3, 12, 200])
def test_select_decoupled_matches_restatement(seed, ncomm):
    rng = np.random.default_rng(100 + seed)
    m = 400
    node = rng.permutation(5000)[:m].astype(np.uint32)
    frm = rng.integers(0, ncomm, m).astype(np.uint32)
    to = rng.integers(0, ncomm, m).astype(np.uint32)
    # coarse gains so that ties occur, a few of them not positive
    gain = rng.integers(-2, 40, m).astype(float) / 8.0
    got = O.select_decoupled(node, frm, to, gain).tolist()
    want = select_moves(node.tolist(), frm.tolist(), to.tolist(), gain.tolist())
    assert got == want
    assert len(want) > 0


def apply_delta(off, col, w, n, ds, dd, dw, delta_n):
    """in_memory.rs:103-137: the existing edges keyed (u, v) with u < v (so
    existing self-loops are dropped), the batch added in batch order on
    (min, max) keys, w > 1e-12 kept, node count the larger of the two; rows
    then built with both directions (a self-loop twice) and, in the canonical
    order the oracle fixes, sorted by neighbour."""
    edges = {}
    for u in range(n):
        for p in range(int(off[u]), int(off[u + 1])):
            v = int(col[p])
            if u < v:
                edges[(u, v)] = float(w[p])
    for a, b, x in zip(ds, dd, dw):
        key = (min(int(a), int(b)), max(int(a), int(b)))
        edges[key] = edges.get(key, 0.0) + float(x)
    nn = max(n, delta_n)
    rows = [[] for _ in range(nn)]
    for (u, v), x in edges.items():
        if x > 1e-12:
            rows[u].append((v, x))
            rows[v].append((u, x))
    noff = np.zeros(nn + 1, np.uint64)
    ncol, nw = [], []
    for u in range(nn):
        rows[u].sort(key=lambda e: e[0])
        ncol += [e[0] for e in rows[u]]
        nw += [e[1] for e in rows[u]]
        noff[u + 1] = len(ncol)
    return noff, np.array(ncol, np.uint32), np.array(nw, np.float64)


@pytest.mark.parametrize("seed", range(5))
@pytest.mark.parametrize("integral", [True, False])
def test_apply_delta_matches_restatement(seed, integral):
    rng = np.random.default_rng(200 + seed)
    n, m = 120, 500
    s = rng.integers(0, n, m)
    t = rng.integers(0, n, m)
    s[:6] = t[:6]  # existing self-loops, which apply_delta drops
    w = rng.integers(1, 4, m).astype(float) if integral else rng.uniform(0.5, 2.0, m)
    g = O.Graph.from_edges(n, s.astype(np.uint32), t.astype(np.uint32), w)
    g = g.apply_delta([], [], [], keep_self_loops=True)  # canonical, duplicates merged
    off, col, ww = g.csr()
    k = 150
    ds = rng.integers(0, n + 10, k)
    dd = rng.integers(0, n + 10, k)
    dw = rng.integers(-3, 4, k).astype(float) if integral else rng.uniform(-2.5, 2.5, k)
    # exact deletes of existing edges, repeated keys, a self-loop in the batch
    for i in range(0, 30, 3):
        u = int(rng.integers(0, n))
        if off[u + 1] > off[u]:
            p = int(rng.integers(off[u], off[u + 1]))
            ds[i], dd[i], dw[i] = u, col[p], -ww[p]
    ds[40:44], dd[40:44] = ds[39], dd[39]
    ds[50], dd[50], dw[50] = 7, 7, 2.5
    delta_n = n + 10
    ref = g.apply_delta(ds.astype(np.uint32), dd.astype(np.uint32), dw, delta_n=delta_n)
    ro, rc, rw = ref.csr()
    eo, ec, ew = apply_delta(off, col, ww, n, ds, dd, dw, delta_n)
    assert np.array_equal(ro, eo) and np.array_equal(rc, ec)
    assert np.array_equal(rw.view(np.uint64), ew.view(np.uint64))


def inc_aggregation(off, col, w, ds, dd, dw, s_pre, s_cur, refined):
    """hit_leiden.rs:1639-1731: ΔG lifted through s_pre; for each refined v
    (ascending) every neighbour j != v with s_cur(j) = s_pre(j) or v < j moves
    its weight from (s_pre v, s_pre j) to (s_cur v, s_cur j); v's self-loop
    weight (both stored copies) moves likewise if above 1e-12; s_pre <- s_cur
    on the refined nodes; records summed per (min, max) key in push order and
    kept if |w| > 1e-9; node count max(s_cur, s_pre) + 1."""
    recs = [(int(s_pre[a]), int(s_pre[b]), float(x)) for a, b, x in zip(ds, dd, dw)]
    for v in np.flatnonzero(refined):
        v = int(v)
        loop = 0.0
        for p in range(int(off[v]), int(off[v + 1])):
            j = int(col[p])
            if j == v:
                loop += float(w[p])
                continue
            if s_cur[j] == s_pre[j] or v < j:
                recs.append((int(s_pre[v]), int(s_pre[j]), -float(w[p])))
                recs.append((int(s_cur[v]), int(s_cur[j]), float(w[p])))
        if abs(loop) > 1e-12:
            recs.append((int(s_pre[v]), int(s_pre[v]), -loop))
            recs.append((int(s_cur[v]), int(s_cur[v]), loop))
    nsp = np.array(s_pre, np.uint32)
    nsp[refined.astype(bool)] = np.asarray(s_cur, np.uint32)[refined.astype(bool)]
    comp = {}
    for a, b, x in recs:
        key = (min(a, b), max(a, b))
        comp[key] = comp.get(key, 0.0) + x
    out = sorted((k, x) for k, x in comp.items() if abs(x) > 1e-9)
    nn = max(int(np.max(s_cur)), int(np.max(s_pre))) + 1
    return out, nsp, nn


@pytest.mark.parametrize("seed", range(5))
@pytest.mark.parametrize("integral", [True, False])
def test_inc_aggregation_matches_restatement(seed, integral):
    rng = np.random.default_rng(300 + seed)
    n, m = 150, 700
    s = rng.integers(0, n, m)
    t = rng.integers(0, n, m)
    s[:8] = t[:8]  # self-loops of the level's nodes
    w = rng.integers(1, 4, m).astype(float) if integral else rng.uniform(0.5, 2.0, m)
    g = O.Graph.from_edges(n, s.astype(np.uint32), t.astype(np.uint32), w)
    g = g.apply_delta([], [], [], keep_self_loops=True)
    off, col, ww = g.csr()
    s_pre = rng.integers(0, 40, n).astype(np.uint32)
    refined = (rng.random(n) < 0.3).astype(np.uint8)
    s_cur = s_pre.copy()
    moved = refined.astype(bool) & (rng.random(n) < 0.7)
    s_cur[moved] = rng.integers(0, 60, int(moved.sum())).astype(np.uint32)
    k = 40
    ds = rng.integers(0, n, k).astype(np.uint32)
    dd = rng.integers(0, n, k).astype(np.uint32)
    dw = rng.integers(-2, 3, k).astype(float) if integral else rng.uniform(-2.0, 2.0, k)
    (u, v, x), nsp, nn = O.inc_aggregation(g, ds, dd, dw, s_pre, s_cur, refined)
    want, wsp, wnn = inc_aggregation(off, col, ww, ds, dd, dw, s_pre, s_cur, refined)
    got = sorted(((int(a), int(b)), float(c)) for a, b, c in zip(u, v, x))
    assert [k_ for k_, _ in got] == [k_ for k_, _ in want]
    assert all(np.float64(a).view(np.uint64) == np.float64(b).view(np.uint64)
               for (_, a), (_, b) in zip(got, want))
    assert np.array_equal(nsp, wsp) and nn == wnn


def inc_movement(off, col, w, n, ds, dd, dw, f, s, gamma, tw, max_rounds=20):
    """hit_leiden.rs:1024-1101 with throughput.rs:80-202: A and K marks from
    the batch (all active for an empty batch); degrees in CSR order and
    community degrees in node order; then up to 20 Jacobi rounds on a snapshot:
    evaluate every active vertex, select decoupled moves, stop on a total gain
    <= 0, apply the moves in selected order, and activate the neighbours of
    moved vertices outside their new community (K marks for same-s pairs).
    2m is the oracle's canonical value, passed in."""
    f = [int(x) for x in f]
    active = [False] * n
    changed = [False] * n
    affected = [False] * n
    for a, b, x in zip(ds, dd, dw):
        a, b = int(a), int(b)
        if x > 0.0 and f[a] != f[b]:
            active[a] = active[b] = True
        if x < 0.0 and f[a] == f[b]:
            active[a] = active[b] = True
        if s[a] == s[b]:
            affected[a] = affected[b] = True
    if len(ds) == 0:
        active = [True] * n
    k = [0.0] * n
    for i in range(n):
        for p in range(int(off[i]), int(off[i + 1])):
            k[i] += float(w[p])
    d = [0.0] * (2 * n + 2)
    for i in range(n):
        d[f[i]] += k[i]
    act = [i for i in range(n) if active[i]]
    it = 0
    while act and it < max_rounds:
        cand = []
        for v in act:
            bt, bg = best_move(off, col, w, v, f, d, k, tw, gamma, n)
            if bg > 0.0:
                cand.append((v, f[v], bt, k[v], bg))
        sel_nodes = select_moves([c[0] for c in cand], [c[1] for c in cand],
                                 [c[2] for c in cand], [c[4] for c in cand])
        by_node = {c[0]: c for c in cand}
        sel = [by_node[v] for v in sel_nodes]
        total = 0.0
        for c in sel:
            total += c[4]
        it += 1
        if total <= 0.0:
            break
        for v, fr, to, kv, _ in sel:
            f[v] = to
            d[fr] -= kv
            d[to] += kv
            changed[v] = True
        nxt = [False] * n
        for v, _, to, _, _ in sel:
            for p in range(int(off[v]), int(off[v + 1])):
                j = int(col[p])
                if f[j] != to:
                    nxt[j] = True
                if s[v] == s[j]:
                    affected[v] = affected[j] = True
        act = [i for i in range(n) if nxt[i]]
    return f, changed, affected, it


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("empty_batch", [False, True])
def test_inc_movement_matches_restatement(seed, integral, empty_batch):
    rng = np.random.default_rng(400 + seed)
    n, m = 200, 900
    s = rng.integers(0, n, m)
    t = rng.integers(0, n, m)
    s[:5] = t[:5]
    w = rng.integers(1, 4, m).astype(float) if integral else rng.uniform(0.5, 2.0, m)
    g = O.Graph.from_edges(n, s.astype(np.uint32), t.astype(np.uint32), w)
    g = g.apply_delta([], [], [], keep_self_loops=True)
    off, col, ww = g.csr()
    tw = g.total_weight() * 2.0
    f = rng.integers(0, 30, n).astype(np.uint32)
    sub = f.copy()
    sub[rng.random(n) < 0.3] += 100  # some sub-communities differ from f
    if empty_batch:
        ds = dd = np.zeros(0, np.uint32)
        dw = np.zeros(0)
    else:
        k = 60
        ds = rng.integers(0, n, k).astype(np.uint32)
        dd = rng.integers(0, n, k).astype(np.uint32)
        dw = np.where(rng.random(k) < 0.8, 1.0, -1.0)
    gf, gch, gaf, git = O.inc_movement(g, ds, dd, dw, f, sub, 1.0, O.MODE_THROUGHPUT,
                                       compact=False)
    wf, wch, waf, wit = inc_movement(off, col, ww, n, ds, dd, dw, f, sub, 1.0, tw)
    assert gf.tolist() == wf and gch.tolist() == wch and gaf.tolist() == waf and git == wit
    assert any(wch)


def _cc_split(off, col, s, verts, visited):
    from collections import deque
    comps = []
    for st in verts:
        if visited[st]:
            continue
        comp, q = [], deque([st])
        visited[st] = True
        while q:
            v = q.popleft()
            comp.append(v)
            sc = s[v]
            for p in range(int(off[v]), int(off[v + 1])):
                j = int(col[p])
                if s[j] == sc and not visited[j]:
                    visited[j] = True
                    q.append(j)
        comps.append(comp)
    return comps


def _refine_split(off, col, w, n, s, affected):
    """The splitting half of inc_refinement (hit_leiden.rs:1265-1357), shared
    by both modes: returns s, the refined flags, sub-community sizes, node
    degrees, sub-community degrees (node order) and the refined nodes sorted
    by degree (stable)."""
    s = [int(x) for x in s]
    refined = [False] * n
    aff = {s[v] for v in range(n) if affected[v]}
    groups = {}
    for i in range(n):
        if s[i] in aff:
            groups.setdefault(s[i], []).append(i)
    nxt = max(s) + 1
    visited = [False] * n
    for sc in sorted(groups):
        verts = groups[sc]
        comps = _cc_split(off, col, s, verts, visited)
        for v in verts:
            visited[v] = False
        if len(comps) <= 1:
            continue
        largest = max(i for i in range(len(comps))
                      if len(comps[i]) == max(len(c) for c in comps))
        for i, comp in enumerate(comps):
            if i == largest:
                continue
            for v in comp:
                s[v] = nxt
                refined[v] = True
            nxt += 1
    if all(s[i] == i for i in range(n)):
        refined = [True] * n
    sizes = {}
    for x in s:
        sizes[x] = sizes.get(x, 0) + 1
    k = [0.0] * n
    for i in range(n):
        for p in range(int(off[i]), int(off[i + 1])):
            k[i] += float(w[p])
    dS = {}
    for i in range(n):
        dS[s[i]] = dS.get(s[i], 0.0) + k[i]
    rs = sorted((i for i in range(n) if refined[i]), key=lambda i: k[i])
    return s, refined, sizes, k, dS, rs


def inc_refinement(off, col, w, n, f, s, affected, gamma, tw, counts=None):
    """hit_leiden.rs:1265-1390 with the throughput merge
    (:1554-1637, throughput.rs:239-359): affected sub-communities split into
    connected components over same-s edges, the largest (the last of equal
    ones) keeping its id and the others taking fresh ids from max(s) + 1; all
    refined when s is the identity; refined nodes by degree (stable); the
    T-filter blocks candidate sub-communities with ΔQ(S→∅) > 1e-9; then every
    refined singleton picks its best same-community neighbour sub-community on
    the snapshot and the moves are applied in list order.  The orders the
    reference leaves to its hash maps are the oracle's canonical ones:
    sub-communities ascending, candidates in first-encounter order."""
    f = [int(x) for x in f]
    s, refined, sizes, k, dS, rs = _refine_split(off, col, w, n, s, affected)
    # T-filter (compute_blocked_subcommunities)
    cands = set()
    for v in rs:
        if sizes[s[v]] != 1:
            continue
        for p in range(int(off[v]), int(off[v + 1])):
            j = int(col[p])
            if f[j] == f[v] and s[j] != s[v]:
                cands.add(s[j])
    dpar = {}
    for i in range(n):
        dpar[f[i]] = dpar.get(f[i], 0.0) + k[i]
    blocked = set()
    for c in cands:
        ds = dS.get(c, 0.0)
        if ds <= 0.0:
            continue
        parent = f[next(i for i in range(n) if s[i] == c)]
        wsp = 0.0
        for i in range(n):
            if s[i] != c:
                continue
            for p in range(int(off[i]), int(off[i + 1])):
                if f[int(col[p])] == parent:
                    wsp += float(w[p])
        dq = -wsp / tw + gamma * ds * (dpar[parent] - ds) / (tw * tw)
        if dq > 1e-9:
            blocked.add(c)
    # Jacobi merges of refined singletons (try_refinement_move)
    upd = []
    for v in rs:
        if sizes[s[v]] != 1:
            continue
        cs, kv = s[v], k[v]
        nbw, wcur = {}, 0.0
        for p in range(int(off[v]), int(off[v + 1])):
            j = int(col[p])
            if f[j] != f[v]:
                continue
            nbw[s[j]] = nbw.get(s[j], 0.0) + float(w[p])
            if s[j] == cs:
                wcur += float(w[p])
        best, bg = cs, 0.0
        for c, wt in nbw.items():
            if c == cs or c in blocked:
                continue
            g = (wt - wcur) / tw + gamma * kv * (dS.get(cs, 0.0) - kv - dS.get(c, 0.0)) / (tw * tw)
            if g > bg:
                best, bg = c, g
        if bg > 0.0:
            upd.append((v, cs, best, kv))
    for v, old, new, kv in upd:
        s[v] = new
        dS[old] = dS.get(old, 0.0) - kv
        dS[new] = dS.get(new, 0.0) + kv
        sizes[old] -= 1
        sizes[new] = sizes.get(new, 0) + 1
    if counts is not None:
        counts["merges"] = counts.get("merges", 0) + len(upd)
        counts["blocked"] = counts.get("blocked", 0) + len(blocked)
    return s, refined


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("initial", [False, True])
def test_inc_refinement_matches_restatement(seed, integral, initial):
    rng = np.random.default_rng(500 + seed)
    n, m = 200, 700
    s_ = rng.integers(0, n, m)
    t = rng.integers(0, n, m)
    s_[:5] = t[:5]
    w = rng.integers(1, 4, m).astype(float) if integral else rng.uniform(0.5, 2.0, m)
    g = O.Graph.from_edges(n, s_.astype(np.uint32), t.astype(np.uint32), w)
    g = g.apply_delta([], [], [], keep_self_loops=True)
    off, col, ww = g.csr()
    tw = g.total_weight() * 2.0
    f = rng.integers(0, 12, n).astype(np.uint32)
    if initial:
        sub = np.arange(n, dtype=np.uint32)
    else:
        sub = (f * 4 + rng.integers(0, 4, n)).astype(np.uint32)
    affected = (rng.random(n) < 0.4).astype(np.uint8)
    counts = {}
    for gamma in (1.0, 0.3):
        gs, gref = O.inc_refinement(g, f, sub, affected, gamma, O.MODE_THROUGHPUT)
        ws, wref = inc_refinement(off, col, ww, n, f, sub, affected, gamma, tw, counts)
        assert gs.tolist() == ws and gref.tolist() == wref, gamma
        assert any(wref)
    assert counts["merges"] > 0 and counts["blocked"] > 0, counts


def test_hit_leiden_one_level_matches_restatement():
    # hit_leiden.rs:936-1018 at one level, the state the reference reaches
    # (state.rs:35-49, an empty graph pushed first as its tests do): per batch
    # apply_delta, inc_movement, inc_refinement; no aggregation, and def_update
    # changes nothing with one level.  Community ids >= n are rank-compacted
    # when movement starts (the oracle's canonical choice where the reference
    # would index out of bounds).
    rng = np.random.default_rng(600)
    n = 150
    st = O.State(n, levels=1, mode=O.MODE_THROUGHPUT)
    st.push_empty_graph(n)
    off = np.zeros(n + 1, np.uint64)
    col = np.zeros(0, np.uint32)
    w = np.zeros(0)
    f = list(range(n))
    s = list(range(n))
    edges = set()
    for b in range(6):
        k = 120 if b == 0 else 40
        ds, dd, dw = [], [], []
        while len(ds) < k:
            a, c = int(rng.integers(0, n)), int(rng.integers(0, n))
            key = (min(a, c), max(a, c))
            if a == c:
                continue
            if key in edges and rng.random() < 0.3:
                ds.append(a), dd.append(c), dw.append(-1.0)  # delete
                edges.discard(key)
            elif key not in edges:
                ds.append(a), dd.append(c), dw.append(float(rng.integers(1, 3)))
                edges.add(key)
        ds = np.array(ds, np.uint32)
        dd = np.array(dd, np.uint32)
        dw = np.array(dw)
        st.hit_leiden(ds, dd, dw)
        off, col, w = apply_delta(off, col, w, n, ds, dd, dw, n)
        if max(f) >= n:
            ids = sorted(set(f))
            f = [ids.index(x) for x in f]
        kdeg = np.array([w[off[i]:off[i + 1]].sum() if off[i + 1] > off[i] else 0.0
                         for i in range(n)])
        tw = O.tree_sum(kdeg)
        f, _, aff, _ = inc_movement(off, col, w, n, ds, dd, dw, f, s, 1.0, tw)
        s, _ = inc_refinement(off, col, w, n, f, s, aff, 1.0, tw)
        go, gc, gw = st.graph(0).csr()
        assert np.array_equal(go, off) and np.array_equal(gc, col)
        assert np.array_equal(gw.view(np.uint64), w.view(np.uint64))
        assert st.get_map(0, O.MAP_F).tolist() == f, b
        assert st.get_map(0, O.MAP_S_CUR).tolist() == s, b
    assert len(set(f)) < n


def test_modularity_matches_exact_restatement():
    # hit_leiden.rs:121-161, Q = (Σ_intra 2w − Σ_C d(C)²/2m) / 2m, evaluated
    # exactly in rationals from the same f64 inputs.  The reference sums
    # Σ_C in hash order, so its value is only defined up to rounding; the
    # oracle (double-double, one final rounding) must lie within 1e-12
    # relative of the exact value, and so must the reference's own float
    # formula with its sums in edge and node order.
    from fractions import Fraction
    rng = np.random.default_rng(700)
    for trial in range(6):
        n, m = 400, 2500
        s = rng.integers(0, n, m)
        t = rng.integers(0, n, m)
        s[:5] = t[:5]
        w = rng.uniform(0.5, 2.0, m) if trial % 2 else rng.integers(1, 4, m).astype(float)
        part = rng.integers(0, 15 + 5 * trial, n).astype(np.uint32)
        deg = [Fraction(0)] * n
        tot = Fraction(0)
        intra = Fraction(0)
        for a, b, x in zip(s.tolist(), t.tolist(), w.tolist()):
            x = Fraction(x)
            deg[a] += x
            deg[b] += x
            tot += x
            if part[a] == part[b]:
                intra += 2 * x
        tm = 2 * tot
        dc = {}
        for i in range(n):
            dc[int(part[i])] = dc.get(int(part[i]), Fraction(0)) + deg[i]
        exact = (intra - sum(v * v / tm for v in dc.values())) / tm
        q = O.modularity_edges(n, s.astype(np.uint32), t.astype(np.uint32), w, part)
        assert abs(Fraction(q) - exact) <= abs(exact) * Fraction(1, 10**12)
        # the reference's float expression, sums in edge / node / id order
        fd = [0.0] * n
        ft = fi = 0.0
        for a, b, x in zip(s.tolist(), t.tolist(), w.tolist()):
            fd[a] += x
            fd[b] += x
            ft += x
            if part[a] == part[b]:
                fi += x * 2.0
        ftm = ft * 2.0
        fc = {}
        for i in range(n):
            fc[int(part[i])] = fc.get(int(part[i]), 0.0) + fd[i]
        fq = (fi - sum(v * v / ftm for v in (fc[c] for c in sorted(fc)))) / ftm
        assert abs(Fraction(fq) - exact) <= abs(exact) * Fraction(1, 10**12)


def inc_movement_deterministic(off, col, w, n, ds, dd, dw, f, s, gamma, tw):
    """hit_leiden.rs:1024-1066 seeding, then the deterministic loop
    (:1103-1191): pop the lowest active vertex; neighbour weights per
    community in CSR order with self-loops counted; strict `>` over the
    candidates in first-encounter order, then the empty community, whose id
    starts at the length of the community-degree array, n, and grows past each
    one used; move, mark B, re-activate neighbours outside the new community,
    K for same-s pairs."""
    f = [int(x) for x in f]
    active = set()
    changed = [False] * n
    affected = [False] * n
    for a, b, x in zip(ds, dd, dw):
        a, b = int(a), int(b)
        if (x > 0.0 and f[a] != f[b]) or (x < 0.0 and f[a] == f[b]):
            active.update((a, b))
        if s[a] == s[b]:
            affected[a] = affected[b] = True
    if len(ds) == 0:
        active = set(range(n))
    k = [0.0] * n
    for i in range(n):
        for p in range(int(off[i]), int(off[i + 1])):
            k[i] += float(w[p])
    d = [0.0] * n
    for i in range(n):
        d[f[i]] += k[i]
    next_empty = len(d)
    while active:
        v = min(active)
        active.discard(v)
        cur, kv = f[v], k[v]
        nbw, wcur = {}, 0.0
        for p in range(int(off[v]), int(off[v + 1])):
            c = f[int(col[p])]
            nbw[c] = nbw.get(c, 0.0) + float(w[p])
            if c == cur:
                wcur += float(w[p])
        best, bg = cur, 0.0
        for c, wt in nbw.items():
            if c == cur:
                continue
            g = (wt - wcur) / tw + gamma * kv * (d[cur] - kv - d[c]) / (tw * tw)
            if g > bg:
                best, bg = c, g
        eg = -wcur / tw + gamma * kv * (d[cur] - kv) / (tw * tw)
        if eg > bg:
            best, bg = next_empty, eg
        if bg <= 0.0:
            continue
        if best >= len(d):
            d += [0.0] * (best + 1 - len(d))
            next_empty = best + 1
        f[v] = best
        changed[v] = True
        d[cur] -= kv
        d[best] += kv
        for p in range(int(off[v]), int(off[v + 1])):
            j = int(col[p])
            if f[j] != best:
                active.add(j)
            if s[v] == s[j]:
                affected[v] = affected[j] = True
    return f, changed, affected


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("gamma", [1.0, 3.0])
def test_deterministic_movement_matches_restatement(seed, gamma):
    rng = np.random.default_rng(800 + seed)
    n, m = 150, 600
    s_ = rng.integers(0, n, m)
    t = rng.integers(0, n, m)
    s_[:5] = t[:5]
    w = rng.uniform(0.5, 2.0, m)
    g = O.Graph.from_edges(n, s_.astype(np.uint32), t.astype(np.uint32), w)
    g = g.apply_delta([], [], [], keep_self_loops=True)
    off, col, ww = g.csr()
    tw = g.total_weight() * 2.0
    f = rng.integers(0, 20, n).astype(np.uint32)
    sub = f.copy()
    ds = rng.integers(0, n, 50).astype(np.uint32)
    dd = rng.integers(0, n, 50).astype(np.uint32)
    dw = np.where(rng.random(50) < 0.8, 1.0, -1.0)
    gf, gch, gaf, _ = O.inc_movement(g, ds, dd, dw, f, sub, gamma, O.MODE_DETERMINISTIC,
                                     compact=False)
    wf, wch, waf = inc_movement_deterministic(off, col, ww, n, ds, dd, dw, f, sub, gamma, tw)
    assert gf.tolist() == wf and gch.tolist() == wch and gaf.tolist() == waf
    assert any(wch)


def inc_refinement_deterministic(off, col, w, n, f, s, affected, gamma, tw):
    """The same splits, then the deterministic merges (hit_leiden.rs:1392-1413,
    :1419-1511): refined singletons in degree order, one at a time on the live
    state; candidates are same-community neighbour sub-communities in
    first-encounter order, skipped by the live T-filter (:1514-1548) with
    d_parent summed over the node's community in node order and w(S, C) over
    S's members in node and CSR order."""
    f = [int(x) for x in f]
    s, refined, sizes, k, dS, rs = _refine_split(off, col, w, n, s, affected)
    for v in rs:
        if sizes[s[v]] != 1:
            continue
        cs, kv, pc = s[v], k[v], f[v]
        nbw, wcur = {}, 0.0
        for p in range(int(off[v]), int(off[v + 1])):
            j = int(col[p])
            if f[j] != pc:
                continue
            nbw[s[j]] = nbw.get(s[j], 0.0) + float(w[p])
            if s[j] == cs:
                wcur += float(w[p])
        dpar = 0.0
        for i in range(n):
            if f[i] == pc:
                dpar += k[i]
        best, bg = cs, 0.0
        for c, wt in nbw.items():
            if c == cs:
                continue
            ds = dS.get(c, 0.0)
            if ds > 0.0:
                wsp = 0.0
                for i in range(n):
                    if s[i] != c:
                        continue
                    for p in range(int(off[i]), int(off[i + 1])):
                        if f[int(col[p])] == pc:
                            wsp += float(w[p])
                if -wsp / tw + gamma * ds * (dpar - ds) / (tw * tw) > 1e-9:
                    continue
            g = (wt - wcur) / tw + gamma * kv * (dS.get(cs, 0.0) - kv - dS.get(c, 0.0)) / (tw * tw)
            if g > bg:
                best, bg = c, g
        if bg > 0.0:
            s[v] = best
            sizes[cs] -= 1
            sizes[best] = sizes.get(best, 0) + 1
            dS[cs] = dS.get(cs, 0.0) - kv
            dS[best] = dS.get(best, 0.0) + kv
    return s, refined


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("initial", [False, True])
def test_deterministic_refinement_matches_restatement(seed, initial):
    rng = np.random.default_rng(900 + seed)
    n, m = 150, 500
    s_ = rng.integers(0, n, m)
    t = rng.integers(0, n, m)
    s_[:5] = t[:5]
    w = rng.uniform(0.5, 2.0, m)
    g = O.Graph.from_edges(n, s_.astype(np.uint32), t.astype(np.uint32), w)
    g = g.apply_delta([], [], [], keep_self_loops=True)
    off, col, ww = g.csr()
    tw = g.total_weight() * 2.0
    f = rng.integers(0, 10, n).astype(np.uint32)
    sub = np.arange(n, dtype=np.uint32) if initial else (f * 4 + rng.integers(0, 4, n)).astype(np.uint32)
    affected = (rng.random(n) < 0.4).astype(np.uint8)
    for gamma in (1.0, 0.3):
        gs, gref = O.inc_refinement(g, f, sub, affected, gamma, O.MODE_DETERMINISTIC)
        ws, wref = inc_refinement_deterministic(off, col, ww, n, f, sub, affected, gamma, tw)
        assert gs.tolist() == ws and gref.tolist() == wref, gamma
