"""Many graphs on one GPU: the batching form (hl_apply_batches) and the serving
form (hl_server_*).

Both run several graphs concurrently, on their own streams, from a pool of
host threads.  The bar is bit-exact: every graph ends in exactly the state the
plain per-graph path (hl_apply_batch) gives for the same batches.  For the
server, "the same batches" are the coalesced batches it reports, replayed one
by one on an identical copy of each graph.  So each result is the same alone
as in the mix.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

hl = importlib.import_module("hit-leiden_b200")
W = importlib.import_module("hit-leiden_b200.workloads")
L = importlib.import_module("hit-leiden_b200._lib")


def _graphs(count, seed, n_lo=400, n_hi=3000, weights=None):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(n_lo, n_hi))
        n, s, d, w, _ = W.planted(n, float(rng.uniform(4, 10)), float(rng.uniform(0.1, 0.4)),
                                  seed * 100 + i, comm_min=5, comm_max=60, weights=weights)
        out.append((n, s, d, w))
    return out


def _load(gr, levels=10):
    n, s, d, w = gr
    return hl.PartitionState.load(hl.GraphInput.from_arrays("g", n, s, d, w),
                                  hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=levels))


def _same(a, b):
    assert a.levels == b.levels
    for p in range(a.levels):
        for which in (L.HL_MAP_COMMUNITY, L.HL_MAP_REFINED, L.HL_MAP_SUB_PREVIOUS,
                      L.HL_MAP_SUB_CURRENT):
            assert np.array_equal(a._map(p, which), b._map(p, which)), (p, which)
        oa, ca, wa = a.supergraph(p)
        ob, cb, wb = b.supergraph(p)
        assert np.array_equal(oa, ob) and np.array_equal(ca, cb)
        assert np.array_equal(wa.view(np.uint64), wb.view(np.uint64))


def _batch(gr, k, seed, weights=None):
    n, s, d, w = gr
    store = W.EdgeStore(n, s, d, w)
    return W.mixed_batch(store, k, 0.8, seed, weights=weights, preferential=False)


@pytest.mark.parametrize("weights", [None, (0.5, 2.0)])
def test_apply_batches_equals_sequential(weights):
    grs = _graphs(6, 3, weights=weights)
    A = [_load(g) for g in grs]
    B = [_load(g) for g in grs]
    for rnd in range(2):
        batches = [_batch(g, int(0.03 * len(g[1])) + 5, 10 * rnd + i, weights)
                   for i, g in enumerate(grs)]
        stats = hl.apply_batches(A, batches, workers=4)
        assert len(stats) == len(A)
        for st, b in zip(B, batches):
            st.apply_batch(*b)
        for a, b in zip(A, B):
            _same(a, b)
    for s in A + B:
        s.close()


def test_apply_batches_rejects_a_handle_twice():
    g = _graphs(1, 5)[0]
    st = _load(g)
    b = _batch(g, 10, 1)
    with pytest.raises(hl.HitLeidenError) as e:
        hl.apply_batches([st, st], [b, b])
    assert e.value.kind == "InvalidInput"
    st.close()


def test_server_results_same_alone_and_in_mix():
    grs = _graphs(4, 7)
    A = [_load(g) for g in grs]
    B = [_load(g) for g in grs]
    rng = np.random.default_rng(11)
    reqs = {}
    with hl.Server(workers=3) as srv:
        ids = [srv.add(s) for s in A]
        for r in range(48):
            gi = int(rng.integers(0, len(grs)))
            u, v, w = _batch(grs[gi], int(rng.integers(2, 40)), 1000 + r)
            rid = srv.submit(ids[gi], u, v, w)
            reqs[rid] = (gi, u, v, w)
        srv.drain()
        done = []
        while True:
            part = srv.poll(cap=64)
            if not part:
                break
            done += part
    assert sorted(d["request_id"] for d in done) == sorted(reqs)
    assert all(d["status"] == 0 for d in done)
    # replay the server's batches, graph by graph, in its order
    per_graph = {}
    for d in done:
        per_graph.setdefault(d["graph"], {}).setdefault(d["batch_seq"], []).append(d)
    coalesced = 0
    for gi, batches in per_graph.items():
        for seq in sorted(batches):
            recs = sorted(batches[seq], key=lambda d: d["request_id"])
            assert len({d["batch_id"] for d in recs}) == 1
            assert recs[0]["batch_requests"] == len(recs)
            coalesced += len(recs) > 1
            parts = [reqs[d["request_id"]] for d in recs]
            u = np.concatenate([p[1] for p in parts])
            v = np.concatenate([p[2] for p in parts])
            w = np.concatenate([p[3] for p in parts])
            assert recs[0]["batch_edges"] == len(u)
            B[gi].apply_batch(u, v, w)
    for a, b in zip(A, B):
        _same(a, b)
    for d in done:
        assert d["latency_ms"] >= d["service_ms"] >= 0.0
    for s in A + B:
        s.close()


def test_server_admission_within_budget_and_rejection():
    import ctypes as C
    grs = _graphs(2, 9)
    A = [_load(g) for g in grs]
    for i, s in enumerate(A):  # first batch: the handles' scratch buffers exist afterwards
        s.apply_batch(*_batch(grs[i], 40, 77 + i))
    resident = 0
    for s in A:
        used, peak = C.c_uint64(), C.c_uint64()
        L.check(L.lib.hl_device_bytes(s._h, C.byref(used), C.byref(peak)))
        resident += used.value
    # a 40-edge request reserves 41 MiB: two fit in flight beside the resident
    # graphs, a third waits for one of them to finish
    per_edge = 1 << 20
    budget = resident + (114 << 20)
    with hl.Server(workers=2, hbm_budget=budget) as srv:
        srv.set_edge_estimate(per_edge)
        ids = [srv.add(s) for s in A]
        rids = []
        for r in range(12):
            u, v, w = _batch(grs[r % 2], 40, 500 + r)
            rids.append(srv.submit(ids[r % 2], u, v, w))
        # a request whose estimate can never fit is rejected, not queued forever
        u, v, w = _batch(grs[0], 40, 999)
        srv.set_edge_estimate(1 << 40)
        big = srv.submit(ids[0], u, v, w)
        srv.drain()
        done = {d["request_id"]: d for d in srv.poll(cap=64)}
    assert set(done) == set(rids) | {big}
    assert all(done[r]["status"] == 0 for r in rids)
    assert done[big]["status"] == L.HL_ERR_OUT_OF_MEMORY
    for s in A:
        s.close()


def test_server_each_request_same_alone_and_in_mix_within_tolerance():
    """Coalescing changes the batches, so the mix is not bit-identical to each
    request applied alone; the bar is |ΔQ| <= 2e-3.  At the end of every
    coalesced batch the graph has seen a prefix of its requests in arrival
    order; a copy that applies those requests one per batch must be within
    2e-3 of the modularity the server reported for that batch."""
    # requests far smaller than their graph, as in the serving configuration
    # (about 0.05 % of a graph's edges each): the path dependence of the
    # incremental result then stays far inside the tolerance
    grs = _graphs(3, 13, n_lo=20000, n_hi=30000)
    A = [hl.PartitionState.load(hl.GraphInput.from_arrays("g", *g),
                                hl.RunConfig(mode=hl.RunMode.Throughput, batch_modularity=True))
         for g in grs]
    C = [_load(g) for g in grs]
    rng = np.random.default_rng(17)
    reqs = {}
    with hl.Server(workers=1) as srv:  # one worker: requests pile up and coalesce
        ids = [srv.add(s) for s in A]
        for r in range(60):
            gi = int(rng.integers(0, len(grs)))
            u, v, w = _batch(grs[gi], int(rng.integers(5, 60)), 2000 + r)
            reqs[srv.submit(ids[gi], u, v, w)] = (gi, u, v, w)
        srv.drain()
        done = []
        while True:
            part = srv.poll(cap=64)
            if not part:
                break
            done += part
    assert all(d["status"] == 0 for d in done)
    batches = {}
    for d in done:
        batches.setdefault((d["graph"], d["batch_seq"]), []).append(d)
    assert any(len(x) > 1 for x in batches.values()), "no request was coalesced"
    worst = 0.0
    for (gi, seq) in sorted(batches):
        recs = sorted(batches[(gi, seq)], key=lambda d: d["request_id"])
        for d in recs:  # alone: one request per batch, in arrival order
            _, u, v, w = reqs[d["request_id"]]
            C[gi].apply_batch(u, v, w)
        q_alone = C[gi].modularity()
        q_mix = recs[0]["modularity"]
        worst = max(worst, abs(q_alone - q_mix))
        assert abs(q_alone - q_mix) <= 2e-3, (gi, seq, q_alone, q_mix)
    for s in A + C:
        s.close()


def test_level_callback_reports_each_settled_level():
    g = _graphs(1, 21, n_lo=2500, n_hi=3000)[0]
    st = _load(g)
    before = [m.copy() for m in st.current_subcommunity_mapping_per_level]
    seen = []
    st.set_level_callback(lambda level, nodes, ids: seen.append((level, nodes, ids)))
    st.apply_batch(*_batch(g, 200, 5))
    st.set_level_callback(None)
    after = st.current_subcommunity_mapping_per_level
    assert [x[0] for x in seen] == list(range(st.levels))
    for level, nodes, ids in seen:
        assert np.all(np.diff(nodes.astype(np.int64)) > 0)
        assert np.array_equal(ids, after[level][nodes])
        old = len(before[level])
        moved = np.nonzero(before[level] != after[level][:old])[0]
        assert np.array_equal(nodes[nodes < old], moved), level
    # off again: no more calls
    n0 = len(seen)
    st.apply_batch(*_batch(g, 50, 6))
    assert len(seen) == n0
    st.close()


def test_server_emits_levels_before_completion():
    grs = _graphs(3, 23)
    A = [_load(g) for g in grs]
    events = []
    with hl.Server(workers=2) as srv:
        srv.set_level_callback(lambda graph, batch, level, nodes, ids:
                               events.append((graph, batch, level, len(nodes))))
        ids = [srv.add(s) for s in A]
        for r in range(12):
            gi = r % len(grs)
            srv.submit(ids[gi], *_batch(grs[gi], 30, 3000 + r))
        srv.drain()
        done = srv.poll(cap=64)
    assert len(done) == 12 and all(d["status"] == 0 for d in done)
    per_batch = {}
    for graph, batch, level, _ in events:
        per_batch.setdefault(batch, []).append(level)
    for d in done:
        levels = per_batch[d["batch_id"]]
        assert levels == list(range(len(levels))) and len(levels) == A[d["graph"]].levels
        assert 0.0 <= d["level0_ms"] <= d["latency_ms"]
    for s in A:
        s.close()
