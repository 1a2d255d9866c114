"""Quality of the incremental result, in the terms of the reference's own
benchmark report (hit_leiden_incremental.rs:513-665): after the updates, the
GPU state's level-0 partition is compared with a from-scratch multilevel Leiden
run on the final graph (the oracle's seeded restatement of run(),
hit_leiden.rs:30-118) by modularity, NMI, purities and largest-community
Jaccard, and with the throughput-mode bootstrap of the final graph by
modularity.  These are quality bounds, not parity: the incremental update and
a fresh run are different algorithms."""
import importlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

hl = importlib.import_module("hit-leiden_b200")
W = importlib.import_module("hit-leiden_b200.workloads")
IO = importlib.import_module("hit-leiden_b200.io")


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_incremental_quality_close_to_fresh_run(seed):
    n, s, d, w = W.config1(seed)
    st = hl.PartitionState.load(hl.GraphInput.from_arrays("c1", n, s, d, w), hl.RunConfig(mode=hl.RunMode.Throughput))
    ex = set(zip(s.tolist(), d.tolist()))
    us, vs = [s], [d]
    for b in range(5):
        u, v, ww = W.uniform_inserts(n, 1000, 100 * seed + b, ex)
        st.apply_batch(u, v, ww)
        ex.update(zip(u.tolist(), v.tolist()))
        us.append(u)
        vs.append(v)
    q_inc = st.modularity()
    part_inc = st.partition()
    fs, fd = np.concatenate(us), np.concatenate(vs)
    # a sequential from-scratch run (the reference's run()) ...
    part_fresh, q_fresh, _ = O.run(n, fs, fd, None, 1.0, 10, 42 + seed)
    # ... and the throughput-mode bootstrap of the same final graph
    boot = O.State(n, mode=O.MODE_THROUGHPUT)
    boot.bootstrap(fs, fd, np.ones(len(fs)), max_levels=10)
    q_boot = boot.modularity(0)
    rep = IO.compare_partitions(part_inc, part_fresh)
    # Measured on these seeds: incremental 0.67-0.70, fresh bootstrap
    # 0.64-0.66, sequential run 0.75; NMI to the run 0.80-0.82 (the reference
    # reports NMI 0.77 between its run() and a fresh igraph Leiden).
    assert q_inc >= q_boot - 0.01, (q_inc, q_boot)
    assert q_fresh - q_inc <= 0.1, (q_inc, q_fresh)
    assert rep.nmi >= 0.7, rep
    assert rep.largest_jaccard >= 0.5, rep
    st.close()


@pytest.mark.parametrize("seed", [0, 1])
def test_rmat_bootstrap_quality_against_run(seed):
    """The GPU bootstrap on the large configuration's shape (R-MAT, scale 16)
    against the oracle's run() (the reference's multilevel_leiden with a
    seeded shuffle, hit_leiden.rs:30-323).  The deterministic-mode bootstrap
    (sequential moves, like run()'s queue) lands within 0.02 of it; the
    throughput-mode bootstrap (Jacobi rounds with decoupled selection) is
    reported beside it and must stay within 0.03."""
    n, bs, bd = W.rmat_torch(16, 16, seed, device="cpu")
    s = bs.numpy().view(np.uint32).copy()
    d = bd.numpy().view(np.uint32).copy()
    _, q_run, _ = O.run(n, s, d, None, 1.0, 10, 42 + seed)
    det = hl.PartitionState.load(hl.GraphInput.from_arrays("r", n, s, d, None),
                                 hl.RunConfig(mode=hl.RunMode.Deterministic))
    thr = hl.PartitionState.load(hl.GraphInput.from_arrays("r", n, s, d, None),
                                 hl.RunConfig(mode=hl.RunMode.Throughput))
    q_det, q_thr = det.modularity(), thr.modularity()
    print(f"R-MAT 16 seed {seed}: run() {q_run:.4f}  deterministic bootstrap {q_det:.4f} "
          f"({det.levels} levels)  throughput bootstrap {q_thr:.4f} ({thr.levels} levels)")
    assert abs(q_det - q_run) <= 0.02
    assert q_run - q_thr <= 0.03
    det.close()
    thr.close()
