"""Writes reference_kats.json: the input/output vectors of the reference
crate's own unit tests for the update path, transcribed from their assertion
blocks (file:line per vector).  The crate is Rust and cannot run here, so these
known answers are its golden vectors.  Where a test asserts a property rather
than a whole output (a neighbour present, a weight near a value), the vector
records exactly that assertion.

    python tests/golden/make_reference_kats.py
"""
import json
import os

T = "src/core/algorithm/hit_leiden.rs"
TRIANGLE = [[0, 1, 1.0], [1, 2, 1.0], [0, 2, 1.0]]
TWO_TRIANGLES = TRIANGLE + [[3, 4, 1.0], [4, 5, 1.0], [3, 5, 1.0]]

KATS = {
    "modularity": [
        {"ref": f"{T}:2186-2201", "n": 3, "edges": TRIANGLE, "part": [0, 0, 0], "q": 0.0},
        {"ref": f"{T}:2203-2217", "n": 3, "edges": TRIANGLE, "part": [0, 1, 2], "q": -1.0 / 3.0},
        {"ref": f"{T}:2219-2235", "n": 6, "edges": TWO_TRIANGLES, "part": [0, 0, 0, 1, 1, 1],
         "q": 0.5},
        {"ref": f"{T}:2237-2248", "n": 3, "edges": [], "part": [0, 1, 2], "q": 0.0},
        {"ref": f"{T}:2250-2272", "n": 2, "edges": [[0, 1, 5.0]], "part": [0, 0], "q": 0.0},
        {"ref": f"{T}:2250-2272", "n": 2, "edges": [[0, 1, 5.0]], "part": [0, 1], "q": -0.5},
    ],
    "select_decoupled": [
        {"ref": "src/core/algorithm/throughput.rs:376-383", "node": [1, 2, 3],
         "from": [10, 20, 30], "to": [20, 10, 40], "gain": [10.0, 9.0, 8.0], "selected": [1, 3]},
        {"ref": "src/core/algorithm/throughput.rs:386-400", "node": [10, 11, 12, 13],
         "from": [1, 1, 4, 2], "to": [2, 3, 2, 5], "gain": [10.0, 9.0, 8.0, 7.0],
         "selected": [10, 11, 12]},
    ],
    "canonicalize": [
        {"ref": f"{T}:2449-2455", "labels": [5, 5, 3, 3, 7], "expected": [0, 0, 1, 1, 2]},
        {"ref": f"{T}:2457-2461", "labels": [0, 0, 1, 1, 2], "expected": [0, 0, 1, 1, 2]},
    ],
    "apply_delta": [
        {"ref": f"{T}:1848-1875", "n": 4, "edges": TRIANGLE, "delta": [[2, 3, 1.0]],
         "neighbours": {"3": {"has": [2]}, "2": {"has": [3]}}, "total_weight_change": 1.0},
        {"ref": f"{T}:1878-1897", "n": 3, "edges": TRIANGLE, "delta": [[0, 2, -1.0]],
         "neighbours": {"0": {"has": [1], "lacks": [2]}}},
    ],
    "inc_aggregation": [
        {"ref": f"{T}:2841-2894", "n": 4, "edges": [[0, 1, 1.0], [1, 2, 1.0], [2, 3, 1.0]],
         "s_pre": [0, 0, 2, 2], "s_cur": [0, 0, 0, 2], "refined": [], "delta": [[0, 2, 5.0]],
         "edge_weights": [[0, 2, 5.0]], "absent_or_zero": [[0, 0]]},
        {"ref": f"{T}:2897-2928", "n": 4, "edges": [[0, 1, 1.0], [2, 3, 1.0]],
         "s_pre": [0, 0, 1, 1], "s_cur": [0, 0, 1, 1], "refined": [],
         "delta": [[0, 2, 3.0], [1, 3, 2.0]], "edge_weights": [[0, 1, 5.0]]},
        {"ref": f"{T}:2931-2958", "n": 4, "edges": [[0, 1, 1.0], [2, 3, 1.0]],
         "s_pre": [0, 0, 1, 1], "s_cur": [0, 0, 1, 1], "refined": [],
         "delta": [[0, 2, 3.0], [0, 3, -3.0]], "absent_or_zero": [[0, 1]]},
        {"ref": f"{T}:2961-2993", "n": 3, "edges": [[0, 1, 1.0], [1, 2, 1.0]],
         "s_pre": [0, 1, 2], "s_cur": [0, 1, 1], "refined": [2], "delta": [],
         "next_s_pre": [0, 1, 1]},
    ],
}

if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(out, "w") as fh:
        json.dump(KATS, fh, indent=1)
        fh.write("\n")
    print("wrote", out)
