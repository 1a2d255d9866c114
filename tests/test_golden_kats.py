"""The oracle against the reference crate's golden vectors
(tests/golden/reference_kats.json, written by make_reference_kats.py from the
crate's own unit tests; each vector cites its file:line).  Tolerances are the
reference's own: 1e-9 on modularity and on weights."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "reference_kats.json")) as fh:
    KATS = json.load(fh)


def _cols(edges):
    if not edges:
        return [], [], []
    u, v, w = zip(*edges)
    return list(u), list(v), [float(x) for x in w]


def _ids(vectors):
    return [v["ref"] for v in vectors]


@pytest.mark.parametrize("kat", KATS["modularity"], ids=_ids(KATS["modularity"]))
def test_modularity(kat):
    q = O.modularity_edges(kat["n"], *_cols(kat["edges"]), kat["part"])
    assert abs(q - kat["q"]) < 1e-9


@pytest.mark.parametrize("kat", KATS["select_decoupled"], ids=_ids(KATS["select_decoupled"]))
def test_select_decoupled(kat):
    sel = O.select_decoupled(kat["node"], kat["from"], kat["to"], kat["gain"])
    assert sel.tolist() == kat["selected"]


@pytest.mark.parametrize("kat", KATS["canonicalize"], ids=_ids(KATS["canonicalize"]))
def test_canonicalize(kat):
    assert O.canonicalize(kat["labels"]).tolist() == kat["expected"]


@pytest.mark.parametrize("kat", KATS["apply_delta"], ids=_ids(KATS["apply_delta"]))
def test_apply_delta(kat):
    g = O.Graph.from_edges(kat["n"], *_cols(kat["edges"]))
    g2 = g.apply_delta(*_cols(kat["delta"]))
    off, col, _ = g2.csr()
    for node, want in kat["neighbours"].items():
        v = int(node)
        nb = col[off[v]:off[v + 1]].tolist()
        assert all(x in nb for x in want.get("has", [])), (v, nb)
        assert not any(x in nb for x in want.get("lacks", [])), (v, nb)
    if "total_weight_change" in kat:
        assert abs(g2.total_weight() - g.total_weight() - kat["total_weight_change"]) < 1e-9


@pytest.mark.parametrize("kat", KATS["inc_aggregation"], ids=_ids(KATS["inc_aggregation"]))
def test_inc_aggregation(kat):
    n = kat["n"]
    g = O.Graph.from_edges(n, *_cols(kat["edges"]))
    refined = np.zeros(n, np.uint8)
    refined[kat["refined"]] = 1
    (u, v, w), nsp, _ = O.inc_aggregation(g, *_cols(kat["delta"]), kat["s_pre"], kat["s_cur"],
                                          refined)
    got = {}
    for a, b, x in zip(u.tolist(), v.tolist(), w.tolist()):
        key = (min(a, b), max(a, b))
        got[key] = got.get(key, 0.0) + x
    for a, b, x in kat.get("edge_weights", []):
        assert abs(got.get((a, b), 0.0) - x) < 1e-9, (a, b, got)
    for a, b in kat.get("absent_or_zero", []):
        assert abs(got.get((a, b), 0.0)) < 1e-8, (a, b, got)
    if "next_s_pre" in kat:
        assert nsp.tolist() == kat["next_s_pre"]


def test_fixture_is_what_the_script_writes():
    # the committed JSON is the generator's output
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_reference_kats", os.path.join(HERE, "golden", "make_reference_kats.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert json.loads(json.dumps(mod.KATS)) == KATS
