"""The multi-GPU form of the path is independent replicas (one graph per rank,
no collective on the data path).  Its host logic — barrier, max of the per-rank
times, whole-job rate — is checked here with two `gloo` ranks on the CPU.  Each
rank applies batches to its own graph (with the CPU oracle standing in for the
GPU) and the ranks agree on the slowest time."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    R = importlib.import_module("hit-leiden_b200.replicas")
    W = importlib.import_module("hit-leiden_b200.workloads")
    from oracle import oracle as O
    rep = R.Replicas("gloo", timeout_s=60)
    # every rank owns a different graph: no data crosses ranks
    n, s, d, w, _ = W.planted(600, 5.0, 0.2, 10 + rank, comm_min=5, comm_max=40)
    st = O.State(n, mode=O.MODE_THROUGHPUT)
    st.bootstrap(s, d, w, max_levels=4)
    rep.barrier()
    ex = set(zip(s.tolist(), d.tolist()))
    steps, k = 3, 50
    for b in range(steps):
        u, v, ww = W.uniform_inserts(n, k, 100 * rank + b, ex)
        st.hit_leiden(u, v, ww)
    local_s = 0.5 + rank  # a per-rank time with a known maximum
    mx = rep.max_over_ranks(local_s)
    rate = rep.whole_job_rate(steps, k, mx)
    rep.barrier()
    out.put((rank, mx, rate, float(st.modularity(0))))
    rep.close()


def test_two_gloo_replicas_agree_on_max_and_rate():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, mx, rate, q_mod in res:
        assert mx == pytest.approx(1.5)
        assert rate == pytest.approx(world * 3 * 50 / 1.5)
        assert -0.5 <= q_mod <= 1.0


def test_single_process_is_a_replica_of_one():
    R = importlib.import_module("hit-leiden_b200.replicas")
    for key in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(key, None)
    rep = R.Replicas("gloo")
    assert rep.world == 1 and rep.dist is None
    rep.barrier()
    assert rep.max_over_ranks(2.5) == 2.5
    assert rep.whole_job_rate(4, 100, 2.0) == pytest.approx(200.0)
    rep.close()
