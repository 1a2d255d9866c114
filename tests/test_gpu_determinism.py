"""Run-to-run determinism on the GPU.  Every kernel of the update path is
either order-free (integral sums, atomics with a fixed final value) or fixes
its order, so identical handles fed identical batches must stay bit-identical;
any data race shows up here as a divergence.  The graphs are larger than the
oracle parity cases so that more blocks run concurrently."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

hl = importlib.import_module("hit-leiden_b200")
W = importlib.import_module("hit-leiden_b200.workloads")
L = importlib.import_module("hit-leiden_b200._lib")
gh = pytest.importorskip("tests.gpu_helpers")


def _state(st):
    out = []
    for p in range(st.levels):
        for which in (L.HL_MAP_COMMUNITY, L.HL_MAP_REFINED, L.HL_MAP_SUB_PREVIOUS,
                      L.HL_MAP_SUB_CURRENT):
            out.append(st._map(p, which).copy())
        off, col, w = st.supergraph(p)
        out += [off.copy(), col.copy(), w.view(np.uint64).copy()]
    return out


@pytest.mark.parametrize("weights", [None, (0.5, 2.0)])
def test_identical_handles_stay_identical(weights):
    n, s, d, w, _ = W.planted(60_000, 24.0, 0.3, 5, comm_min=20, comm_max=2000,
                              weights=weights)
    handles = [hl.PartitionState.load(hl.GraphInput.from_arrays("g", n, s, d, w),
                                      hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=10)) for _ in range(3)]
    ref = _state(handles[0])
    for h in handles[1:]:
        assert all(np.array_equal(a, b) for a, b in zip(ref, _state(h)))
    store = W.EdgeStore(n, s, d, w)
    for b in range(3):
        u, v, ww = W.mixed_batch(store, 3000, 0.9, 40 + b, weights=weights)
        store.apply(u, v, ww)
        for h in handles:
            h.apply_batch(u, v, ww)
        ref = _state(handles[0])
        for h in handles[1:]:
            got = _state(h)
            assert len(got) == len(ref)
            assert all(np.array_equal(a, b) for a, b in zip(ref, got)), f"batch {b}"
    for h in handles:
        h.close()


@pytest.mark.parametrize("integral", [True, False])
def test_refinement_repeatable(integral):
    rng = np.random.default_rng(17)
    n = 20_000
    src, dst, w = gh.random_graph(rng, n, 120_000, integral)
    from oracle import oracle as O
    g = O.Graph.from_edges(n, src, dst, w).apply_delta([], [], [], keep_self_loops=True)
    f = gh.random_partition(rng, n, 40)
    s0 = (f * 7 + rng.integers(0, 7, n)).astype(np.uint32)
    aff = rng.random(n) < 0.5
    first = gh.inc_refinement(g, f, s0.copy(), aff, 1.0, True)
    for _ in range(4):
        again = gh.inc_refinement(g, f, s0.copy(), aff, 1.0, True)
        assert np.array_equal(first[0], again[0]) and np.array_equal(first[1], again[1])
