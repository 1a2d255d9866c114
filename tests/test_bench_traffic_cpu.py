"""The bench's roofline.traffic comes from the committed ncu summary of its
own configuration (profiles/move_eval_traffic_<config>.json), never from
another configuration's."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("hl_bench_traffic", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_ratio_per_configuration():
    b = _bench()
    r = b.committed_traffic("rmat25")
    assert r["config"] == "rmat25" and 1.0 < r["traffic_per_algorithmic_byte"] < 10.0
    assert abs(r["traffic_per_algorithmic_byte"] - r["dram_bytes"] / r["algorithmic_bytes"]) < 1e-3
    l = b.committed_traffic("lfr1m")
    assert l["config"] == "lfr1m"
    assert b.committed_traffic("batch256") is None
