"""Round-to-round hub key sums, checked in the oracle.

Between two throughput movement rounds only the moved vertices' labels
change, so the per-key weight sums of a long row can be kept and corrected by
its moved neighbours instead of being recomputed (exact for integral
weights).  With FLAG_HUB_CHECK the oracle evaluates every active row of more
than 512 entries that way as well, with the first CSR position of a key
recomputed only when a key that lost its first entry ties the best gain, and
compares each result with the full evaluation (parallel_frontier.rs:133-239).
The update's results do not depend on the flag."""
import importlib.util
import os

import numpy as np

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _workloads():
    spec = importlib.util.spec_from_file_location("hl_wl_hubcheck",
                                                  os.path.join(ROOT, "hit-leiden_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rmat(scale, seed):
    import torch
    W = _workloads()
    n, s, d = W.rmat_torch(scale, 16, seed, device="cpu")
    k = 1_000_000 >> (25 - scale)
    u, v, w = W.rmat_batch_torch(scale, s, d, k, 0.9, 10_000 + seed)
    as_u32 = lambda x: x.numpy().view(np.uint32).copy()
    return n, as_u32(s), as_u32(d), as_u32(u), as_u32(v), w.numpy().copy()


def test_hub_key_sums_match_full_evaluation():
    O.load()
    n, s, d, u, v, w = _rmat(15, 3)
    states = []
    for flags in (O.FLAG_HUB_CHECK, 0):
        st = O.State(n, levels=1, mode=O.MODE_THROUGHPUT, flags=flags)
        st.bootstrap(s, d, None, max_levels=3)
        O.hub_check_counters()  # the bootstrap's movement is not checked
        st.hit_leiden(u, v, w)
        states.append(st)
        if flags:
            c = O.hub_check_counters()
    assert c["evals"] > 500 and c["builds"] > 0 and c["corrections"] > 0
    assert c["mismatches"] == 0, c
    # the flag changes nothing in the update itself
    for lv in range(states[0].levels):
        assert np.array_equal(states[0].get_map(lv, O.MAP_F), states[1].get_map(lv, O.MAP_F))


def test_stale_first_position_is_recomputed_at_a_tie():
    # a key loses its first entry to a move, then ties the best gain: its true
    # first position decides, and the evaluation still matches the full one
    assert O.hub_check_selftest() == 1
