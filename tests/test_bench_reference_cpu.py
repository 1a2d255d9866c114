"""bench.py's reference arm runs on the CPU alone: its JSON line (the
contract's keys, `impl: reference`, the CPU baseline it describes) and the
faithful variants (the reference's quadratic refinement scans on all host
threads, and the deterministic mode on one) with the reference benchmark's
from-scratch run() per batch, on the small configuration."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*extra):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--config", "ca_hepth", "--steps", "2", "--warmup", "1", *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _run()
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == "edge_updates_per_s"
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert "cpu_variants" not in d


def test_reference_arm_faithful_variants():
    d = _run("--cpu-variants", "--cpu-cap", "120")
    v = d["cpu_variants"]
    ft, fd, sr = v["faithful_throughput"], v["faithful_deterministic"], v["static_run_per_batch"]
    assert ft["value"] > 0 and ft["same_result"] is True
    assert fd["value"] > 0 and fd["cores"] == 1
    assert sr["value"] > 0 and 0.0 < sr["modularity"] < 1.0


def _maps_after_reference_arm(*argv):
    """Run the reference arm in this interpreter's child and report whether
    libhl.so was mapped into it at the end."""
    code = ("import runpy, sys, json\n"
            f"sys.argv = {['bench.py', '--impl', 'reference', *argv]!r}\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('LIBHL_MAPPED', 'libhl.so' in maps)\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][0])
    mapped = [ln for ln in r.stdout.splitlines() if ln.startswith("LIBHL_MAPPED")][0]
    return line, mapped.endswith("True")


def test_reference_arm_never_loads_the_gpu_library():
    line, mapped = _maps_after_reference_arm("--config", "ca_hepth", "--steps", "1",
                                             "--warmup", "0")
    assert line["impl"] == "reference"
    assert not mapped


def test_reference_arm_rmat_stand_in():
    # the R-MAT configuration's CPU sample: the same generator at a small scale
    line, mapped = _maps_after_reference_arm("--config", "rmat25", "--steps", "2", "--warmup",
                                             "1", "--rmat-sample-scale", "12")
    assert not mapped
    assert line["steps"] == 2 and line["warmup"] == 1 and line["value"] > 0
    assert "scale 12 stand-in" in line["cpu_baseline"]["sample"]
    assert line["config"]["batch_edges"] == 1_000_000
