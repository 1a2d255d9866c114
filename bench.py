#!/usr/bin/env python3
"""Benchmark of the HIT-Leiden incremental update path on B200.

One step = one edge-update batch applied through the public C ABI
(hl_apply_batch: G ⊕ ΔG, then inc-movement, inc-refinement and
inc-aggregation on every level, then the top-down level maps) on a graph
resident in HBM, followed by a read-back of the level-0 community map.

Default workload (the large plain-method configuration, the one the target
is stated on): R-MAT scale 25 (33.5M vertices), edge factor 16,
(a,b,c,d) = (.57,.19,.19,.05), symmetrised, duplicates and self-loops
removed (~524M undirected edges), unit weights summed in FP64; batches of 1M
updates (90% R-MAT-sampled inserts, 10% uniform deletes).  Synthetic and
seeded: the reference's datasets are not available.  `--config lfr1m` runs
the mid-size configuration (LFR-style, 1M vertices / ~20M f64 edges, 10k
batches), whose CPU sample also checks full-size bit-exact parity.

Reported (the same K timed batches give both numbers):
  value   edge-updates/s from the device time of each batch (CUDA events on
          the library's stream, from the batch resident in HBM to the end of
          the update), summed over the K steps, max over ranks;
  e2e     edge-updates/s on the host clock around the same calls: the
          host→device copy of the pinned host batch, the update and a
          device→host read of the level-0 community map into pinned memory;
  roofline for the inc-movement evaluation kernels (algorithmic bytes / event
          time), roofline_aggregation for inc-aggregation;
  cpu_baseline: the CPU oracle (a C++ port of the reference's Rust, its
          snapshot evaluations on all host threads as the reference's rayon
          pool) on a bounded sample (see each configuration).

--impl reference runs that CPU port alone, never loading libhl.so.
Multi-GPU (--gpus N under torchrun): independent replicas, one graph per GPU,
no collective on the data path; the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# R-MAT stand-in for the CPU port: the port cannot bootstrap scale 25 (about
# 1B adjacency entries) within the bench's few-minute bound, so its sample is
# the same generator at scale 20 with batches scaled by the same factor.
RMAT_SAMPLE_SCALE = 20


def _module(name):
    """One host-side module of the package, loaded by path without running the
    package's __init__ (which maps libhl.so): the CPU arms must not load the
    GPU library."""
    import importlib.util
    key = "hl_bench_" + name
    if key in sys.modules:
        return sys.modules[key]
    path = os.path.join(ROOT, "hit-leiden_b200", name + ".py")
    spec = importlib.util.spec_from_file_location(key, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[key] = mod
    spec.loader.exec_module(mod)
    return mod

CONFIGS = {
    "lfr1m": {
        "workload": "LFR-style planted graph, 1M vertices / ~20M edges, f64 weights U[0.5,2], "
                    "batches of 10k updates (90% degree-preferential inserts, 10% deletes)",
        "batch": 10000,
    },
    "batch256": {
        "workload": "batching form: 256 independent planted graphs, vertices log-uniform "
                    "[1k, 200k], mu log-uniform [0.1, 0.4], target mean degree U[4, 32], unit "
                    "weights; per graph a batch of 1-5% of its edges (80% inserts, 20% deletes)",
        "batch": 0,
    },
    "serve32": {
        "workload": "serving form: 32 resident planted graphs, vertices log-uniform [100k, 5M] "
                    "(x scale), mu 0.25, target mean degree 16; Poisson request arrivals at "
                    "100 / 1,000 / 10,000 req/s, request sizes log-uniform [10, 100k] edges "
                    "(85% inserts, 15% deletes), 120 GB admission budget",
        "batch": 0,
    },
    "rmat25": {
        "workload": "R-MAT scale 25 (33.5M vertices), edge factor 16, (a,b,c,d) = "
                    "(.57,.19,.19,.05), symmetrised, duplicates and self-loops removed; unit "
                    "weights summed in FP64; batches of 1M updates (90% R-MAT inserts, 10% "
                    "uniform deletes)",
        "batch": 1_000_000,
    },
    "ca_hepth": {
        "workload": "planted graph shaped like ca-HepTh: 9,877 vertices / ~21.8k unit edges, "
                    "mu 0.15, triangle closure; batches of 1,000 uniform inserts",
        "batch": 1000,
    },
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="rmat25")
    ap.add_argument("--levels", type=int, default=10)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-sample-batches", type=int, default=3)
    ap.add_argument("--cpu-sample-cap", type=float, default=45.0,
                    help="wall-clock seconds the CPU sample's timed batches may take "
                         "(at least one batch runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-variants", action="store_true",
                    help="reference arm: also time the faithful CPU variants (the "
                         "reference's quadratic refinement scans; throughput on all host "
                         "threads and deterministic on one) and a from-scratch run() on "
                         "the updated graph, one batch each under --cpu-cap")
    ap.add_argument("--cpu-cap", type=float, default=120.0,
                    help="wall-clock cap in seconds for each faithful variant's batch")
    ap.add_argument("--no-served", action="store_true",
                    help="rmat25: skip the serving-form phase after the timed steps")
    ap.add_argument("--served-requests", type=int, default=48,
                    help="rmat25: requests of the serving-form phase")
    ap.add_argument("--rmat-sample-scale", type=int, default=RMAT_SAMPLE_SCALE,
                    help="R-MAT scale of the CPU port's stand-in sample for rmat25")
    ap.add_argument("--cpu-variant-run", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-variant-mode", default="throughput", help=argparse.SUPPRESS)
    ap.add_argument("--ncu-small", action="store_true",
                    help="small case for ncu captures (rmat25: R-MAT scale 20 with 1M/32-update "
                         "batches; lfr1m: 200k vertices)")
    ap.add_argument("--workers", type=int, default=16,
                    help="host worker threads of the batching / serving forms")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="vertex-count scale of the serving form's graphs")
    ap.add_argument("--requests", type=int, default=400,
                    help="requests per arrival rate in the serving form")
    return ap.parse_args()


def make_graph(cfg_name, seed, small=False):
    W = _module("workloads")
    if cfg_name == "lfr1m":
        if small:
            n, s, d, w = W.config2(seed, n=200_000)
        else:
            n, s, d, w = W.config2(seed)
        return n, s, d, w, (0.5, 2.0), 0.9, True
    n, s, d, w = W.config1(seed)
    return n, s, d, w, None, 1.0, False


def make_batches(n, s, d, w, weights, insert_frac, preferential, count, k, seed):
    W = _module("workloads")
    store = W.EdgeStore(n, s, d, w)
    out = []
    for i in range(count):
        if insert_frac >= 1.0 and not preferential:
            ex = None
            u, v, ww = W.uniform_inserts(n, k, seed * 1000 + i, ex)
            store.apply(u, v, ww)
        else:
            u, v, ww = W.mixed_batch(store, k, insert_frac, seed * 1000 + i, weights=weights,
                                     preferential=preferential)
        out.append((u.astype(np.uint32), v.astype(np.uint32), ww.astype(np.float64)))
    return out


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}", "--format=csv,noheader",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                mx = max(mx, float(parts[2].split()[0]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        j = json.load(open(p))
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(config=None):
    """DRAM bytes per algorithmic byte of the movement evaluation from the
    committed ncu summary of `config` (profiles/move_eval_traffic_<config>.json,
    else the older single-configuration file), scaled to the bench's launch."""
    names = ([f"move_eval_traffic_{config}.json"] if config else []) + ["move_eval_traffic.json"]
    for name in names:
        p = os.path.join(ROOT, "profiles", name)
        if os.path.exists(p):
            try:
                tr = json.load(open(p))
            except Exception:
                continue
            if config is None or tr.get("config") == config:
                return tr
    return None


def export_state(st):
    """Per-level CSR and maps of a GPU state, for the CPU oracle."""
    levels = []
    subs_pre = st.previous_subcommunity_mapping_per_level
    subs_cur = st.current_subcommunity_mapping_per_level
    fs = st.community_mapping_per_level
    gs = st.refined_community_mapping_per_level
    for p in range(st.levels):
        off, col, w = st.supergraph(p)
        levels.append({"off": off, "col": col, "w": w, "f": fs[p], "g": gs[p],
                       "s_pre": subs_pre[p], "s_cur": subs_cur[p]})
    return levels


def cpu_baseline(st, batches, max_batches, cap_s):
    """Time the oracle port on the next batches from the GPU's state (at least
    one, then more while the timed total stays under cap_s); check that the
    GPU state after the same batches is identical (full-size parity)."""
    from oracle import oracle as O
    O.load()
    ora = O.State(st.node_count, levels=1, mode=O.MODE_THROUGHPUT)
    ora.import_levels(export_state(st))
    per = []
    edges = 0
    for (u, v, w) in batches[:max_batches]:
        t0 = time.perf_counter()
        ora.hit_leiden(u, v, w)
        per.append(time.perf_counter() - t0)
        edges += len(u)
        st.apply_batch(u, v, w)
        if sum(per) >= cap_s:
            break
    same = st.levels == ora.levels and all(
        np.array_equal(st.community_mapping_per_level[p], ora.get_map(p, O.MAP_F))
        and np.array_equal(st.current_subcommunity_mapping_per_level[p],
                           ora.get_map(p, O.MAP_S_CUR))
        for p in range(ora.levels))
    q_gpu = st.modularity()
    q_cpu = ora.modularity(0)
    return {"value": edges / sum(per), "seconds": sum(per), "batches": len(per), "edges": edges,
            "batch_s": per, "parity_bit_exact": bool(same), "dq": abs(q_gpu - q_cpu),
            "threads": O.num_threads()}


def rmat_sample(seed, scale=RMAT_SAMPLE_SCALE):
    """The CPU port's R-MAT stand-in (scale RMAT_SAMPLE_SCALE, same generator
    and parameters as the full workload, generated with torch on the host)."""
    W = _module("workloads")
    n, s, d = W.rmat_torch(scale, 16, seed, device="cpu")
    k = 1_000_000 >> (25 - scale)

    def batch(i):
        u, v, w = W.rmat_batch_torch(scale, s, d, k, 0.9, 10_000 + i)
        return (u.numpy().view(np.uint32).copy(), v.numpy().view(np.uint32).copy(),
                w.numpy().copy())
    return (n, s.numpy().view(np.uint32).copy(), d.numpy().view(np.uint32).copy(), k, batch)


def cpu_rmat_sample(seed, levels, warm, max_batches, cap_s, scale=RMAT_SAMPLE_SCALE):
    """Bootstrap the oracle on the R-MAT stand-in (untimed), apply `warm`
    batches untimed, then time batches until max_batches or cap_s."""
    from oracle import oracle as O
    O.load()
    n, s, d, k, batch = rmat_sample(seed, scale)
    st = O.State(n, mode=O.MODE_THROUGHPUT)
    t0 = time.perf_counter()
    st.bootstrap(s, d, None, max_levels=levels)
    boot = time.perf_counter() - t0
    i = 0
    for _ in range(warm):
        st.hit_leiden(*batch(i))
        i += 1
    per = []
    while len(per) < max_batches:
        b = batch(i)
        i += 1
        t0 = time.perf_counter()
        st.hit_leiden(*b)
        per.append(time.perf_counter() - t0)
        if sum(per) >= cap_s:
            break
    return {"value": len(per) * k / sum(per), "batches": len(per), "batch_edges": k,
            "batch_s": per, "bootstrap_s": boot, "warmup": warm, "vertices": n,
            "edges": int(len(s)), "levels": st.levels, "modularity": st.modularity(0),
            "threads": O.num_threads(), "scale": scale}


def _rmat_sample_text(r):
    return (f"R-MAT scale {r['scale']} stand-in for scale 25 ({r['vertices']} vertices, "
            f"{r['edges']} edges, same generator and (a,b,c,d); batches of {r['batch_edges']} "
            f"= 1M/{1 << (25 - r['scale'])} updates, 90% R-MAT inserts / 10% deletes): "
            f"untimed bootstrap ({r['bootstrap_s']:.1f} s, {r['levels']} levels) and "
            f"{r['warmup']} untimed batch(es), then {r['batches']} timed batch(es) "
            f"(median {statistics.median(r['batch_s']):.2f} s, min {min(r['batch_s']):.2f}, "
            f"max {max(r['batch_s']):.2f}) on {r['threads']} host threads.  The port cannot "
            f"bootstrap scale 25 within the bench's bound; its per-update work grows with the "
            f"graph (apply_delta rewrites every row), so the stand-in overstates the CPU rate "
            f"at scale 25")


def _oracle_levels(st):
    """Per-level CSR and maps of an oracle state (the form import_levels takes)."""
    from oracle import oracle as O
    levels = []
    for p in range(st.levels):
        off, col, w = st.graph(p).csr()
        levels.append({"off": off, "col": col, "w": w, "f": st.get_map(p, O.MAP_F),
                       "g": st.get_map(p, O.MAP_G), "s_pre": st.get_map(p, O.MAP_S_PRE),
                       "s_cur": st.get_map(p, O.MAP_S_CUR)})
    return levels


def run_cpu_variant(args):
    """One faithful variant on one batch, from a state saved by the reference
    arm: import it with the reference's quadratic refinement scans, time the
    batch, print a JSON line."""
    from oracle import oracle as O
    O.load()
    z = np.load(args.cpu_variant_run)
    P = int(z["levels"])
    levels = [{k: z[f"{k}{p}"] for k in ("off", "col", "w", "f", "g", "s_pre", "s_cur")}
              for p in range(P)]
    if args.cpu_variant_mode == "run":
        # the reference benchmark's own operation: a from-scratch run() on the
        # graph after the batch (hit_leiden.rs:30-118)
        off, col, w = z["off0"], z["col0"], z["w0"]
        n = len(off) - 1
        rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off).astype(np.int64))
        keep = rows < col
        g = O.Graph.from_edges(n, rows[keep], col[keep], w[keep])
        off2, col2, w2 = g.apply_delta(z["u"], z["v"], z["w_batch"]).csr()
        rows2 = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off2).astype(np.int64))
        keep2 = rows2 < col2
        t0 = time.perf_counter()
        _, q, _ = O.run(n, rows2[keep2], col2[keep2], w2[keep2])
        t = time.perf_counter() - t0
        print(json.dumps({"seconds": t, "threads": 1, "modularity": q}), flush=True)
        return
    det = args.cpu_variant_mode == "deterministic"
    if det:
        O.set_num_threads(1)
    flags = O.FLAG_FAITHFUL_SCANS | (O.FLAG_MULTILEVEL if P > 1 else 0)
    st = O.State(len(levels[0]["f"]), levels=1,
                 mode=O.MODE_DETERMINISTIC if det else O.MODE_THROUGHPUT)
    st.import_levels(levels, flags=flags)
    t0 = time.perf_counter()
    st.hit_leiden(z["u"], z["v"], z["w_batch"])
    t = time.perf_counter() - t0
    print(json.dumps({"seconds": t, "threads": O.num_threads(),
                      "modularity": st.modularity(0)}), flush=True)


def _time_variants(st, batch, k, cap):
    """Save the bootstrapped state and the batch, then run each faithful variant
    in a child process killed at `cap` seconds (plus a little for loading)."""
    out = {}
    u, v, ww = batch
    with tempfile.TemporaryDirectory() as td:
        levels = _oracle_levels(st)
        arrays = {"levels": len(levels), "u": u, "v": v, "w_batch": ww}
        for p, lv in enumerate(levels):
            arrays.update({f"{kk}{p}": a for kk, a in lv.items()})
        path = os.path.join(td, "state.npz")
        np.savez(path, **arrays)
        del levels, arrays
        for name, mode in (("faithful_throughput", "throughput"),
                           ("faithful_deterministic", "deterministic"),
                           ("static_run_per_batch", "run")):
            det = mode != "throughput"
            cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                   "--cpu-variant-run", path, "--cpu-variant-mode", mode]
            try:
                r = subprocess.run(cmd, capture_output=True, text=True, timeout=cap + 30.0)
                res = json.loads(r.stdout.strip().splitlines()[-1])
                out[name] = {"value": k / res["seconds"], "unit": "edge-updates/s",
                             "seconds": res["seconds"], "cores": res["threads"],
                             "modularity": res["modularity"]}
            except subprocess.TimeoutExpired:
                out[name] = {"dnf_after_s": cap, "cores": 1 if det else None}
    return out


def run_reference(args, cfg):
    """CPU port of the reference path alone (libhl.so is never loaded).  It
    bootstraps untimed, applies --warmup batches untimed and then times up to
    --steps batches of the same stream, stopping early once --cpu-cap seconds
    of timed batches have run (at least one runs)."""
    from oracle import oracle as O
    O.load()
    if args.config == "rmat25":
        r = cpu_rmat_sample(args.seed, args.levels, min(args.warmup, 1), args.steps,
                            args.cpu_cap, args.rmat_sample_scale)
        val = r["value"]
        steps, warm, k = r["batches"], r["warmup"], r["batch_edges"]
        ms = 1000.0 * sum(r["batch_s"]) / steps
        sample = _rmat_sample_text(r)
        q, levels = r["modularity"], r["levels"]
        config = {"workload": cfg["workload"], "scale": 25, "batch_edges": cfg["batch"]}
    else:
        n, s, d, w, wts, ins, pref = make_graph(args.config, args.seed, args.ncu_small)
        k = cfg["batch"]
        batches = make_batches(n, s, d, w, wts, ins, pref, args.warmup + args.steps, k,
                               args.seed)
        st = O.State(n, mode=O.MODE_THROUGHPUT)
        if args.levels > 1:
            st.bootstrap(s, d, w, max_levels=args.levels)
        else:
            st = O.State(n, levels=1, mode=O.MODE_THROUGHPUT)
            st.push_empty_graph()
            st.hit_leiden(s, d, w)
        for (u, v, ww) in batches[:args.warmup]:
            st.hit_leiden(u, v, ww)
        variants = (_time_variants(st, batches[args.warmup], k, args.cpu_cap)
                    if args.cpu_variants else None)
        per = []
        q_first = None
        for (u, v, ww) in batches[args.warmup:]:
            t0 = time.perf_counter()
            st.hit_leiden(u, v, ww)
            per.append(time.perf_counter() - t0)
            if variants is not None and q_first is None:
                q_first = st.modularity(0)
            if sum(per) >= args.cpu_cap:
                break
        steps, warm = len(per), args.warmup
        val = steps * k / sum(per)
        ms = 1000.0 * sum(per) / steps
        sample = (f"batches {warm}..{warm + steps - 1} of the stream ({k} updates each) after "
                  f"an untimed bootstrap and {warm} untimed batches, the same batch indices the "
                  f"GPU arm times first (median {statistics.median(per):.2f} s a batch; "
                  "snapshot evaluations on all host threads, up to 64)")
        q, levels = st.modularity(0), st.levels
        config = {"workload": cfg["workload"], "vertices": n, "edges": int(len(s)),
                  "batch_edges": k}
        if variants is not None and "modularity" in variants["faithful_throughput"]:
            # the faithful scans change the cost, not the result
            variants["faithful_throughput"]["same_result"] = (
                variants["faithful_throughput"]["modularity"] == q_first)
    line = {
        "impl": "reference", "metric": "edge_updates_per_s", "value": val,
        "unit": "edge-updates/s", "n_gpus": args.gpus, "steps": steps, "warmup": warm,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
        "cpu_baseline": {"value": val, "unit": "edge-updates/s", "cores": O.num_threads(),
                         "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": "edge-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "modularity": q, "levels": levels,
    }
    if args.config != "rmat25" and variants is not None:
        line["cpu_variants"] = variants
    print(json.dumps(line), flush=True)


def _load_many(hl, graphs, levels, device, threads=16):
    """Load and bootstrap many graphs concurrently (each on its own stream)."""
    from concurrent.futures import ThreadPoolExecutor

    def one(g):
        n, s, d, w = g
        return hl.PartitionState.load(hl.GraphInput.from_arrays("g", n, s, d, w),
                                      hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=levels, device=device))
    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(one, graphs))


def run_batching(args, cfg):
    """Batching form: every step applies one batch to each of 256 graphs, once
    through hl_apply_batches (graphs concurrent) and once through the plain
    per-graph path (a loop of hl_apply_batch) on an identical copy; both from
    host arrays, host clock with the device synchronised on both sides."""
    import torch
    R = importlib.import_module("hit-leiden_b200.replicas")
    W = _module("workloads")
    rep = R.Replicas("nccl")
    torch.cuda.set_device(rep.local)
    hl = importlib.import_module("hit-leiden_b200")
    graphs = W.config4(args.seed + rep.rank)
    rng = np.random.default_rng(args.seed + 7)
    fracs = rng.uniform(0.01, 0.05, len(graphs))
    A = _load_many(hl, graphs, args.levels, rep.local)
    B = _load_many(hl, graphs, args.levels, rep.local)

    def batches(step):
        out = []
        for i, (n, s, d, w) in enumerate(graphs):
            k = max(1, int(fracs[i] * len(s)))
            out.append(W.fast_batch(n, s, d, k, 0.8, (step + 1) * 1_000_003 + i))
        return out
    K, Wm = args.steps, args.warmup
    t_plain = t_batch = 0.0
    edges = 0
    launches = 0
    for step in range(Wm + K):
        bs = batches(step)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for st, b in zip(B, bs):
            st.apply_batch(*b)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        stats = hl.apply_batches(A, bs, workers=args.workers)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if step >= Wm:
            t_plain += t1 - t0
            t_batch += t2 - t1
            edges += sum(len(b[0]) for b in bs)
            launches += sum(x.launches for x in stats)
    same = all(np.array_equal(a.community_mapping_per_level[0], b.community_mapping_per_level[0])
               for a, b in zip(A, B))
    t_batch = rep.max_over_ranks(t_batch)
    t_plain = rep.max_over_ranks(t_plain)
    value = rep.world * edges / t_batch
    plain = rep.world * edges / t_plain
    if rep.rank == 0:
        line = {
            "metric": "edge_updates_per_s", "value": value, "unit": "edge-updates/s",
            "n_gpus": rep.world, "steps": K, "warmup": Wm, "ms_per_step": 1000.0 * t_batch / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": cfg["workload"], "graphs": len(graphs),
                       "vertices": int(sum(g[0] for g in graphs)),
                       "edges": int(sum(len(g[1]) for g in graphs)),
                       "edges_per_step": edges // K, "workers": args.workers,
                       "parallelism": f"replicas{rep.world}",
                       "timing": "host clock, device synchronised on both sides",
                       "plain_gpu_edge_updates_per_s": plain, "batched_over_plain": value / plain,
                       "batched_equals_plain_bit_exact": bool(same)},
            "e2e": {"value": value, "unit": "edge-updates/s",
                    "h2d_bytes_per_step": int(16 * edges // K), "d2h_bytes_per_step": 0},
            "gpu_launches": int(launches), "roofline": None, "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    for st in A + B:
        st.close()
    rep.close()


def _serve(hl, states, reqs, arrivals, workers, coalesce, budget):
    """Submit reqs[i] = (graph, u, v, w) at arrivals[i] seconds; return the
    completion records and the wall time from the first submit to the last
    completion."""
    srv = hl.Server(workers=workers, hbm_budget=budget)
    if coalesce is not None:
        srv.set_coalescing(coalesce)
    # per-level output on: the records then say when each batch's level 0
    # was settled (level0_ms), the point a pipeline can start summarising
    srv.set_level_callback(lambda graph, batch, level, nodes, ids: None)
    ids = [srv.add(s) for s in states]
    t0 = time.perf_counter()
    for (g, u, v, w), ta in zip(reqs, arrivals):
        while True:
            dt = ta - (time.perf_counter() - t0)
            if dt <= 0:
                break
            if dt > 0.002:
                time.sleep(dt - 0.001)
        srv.submit(ids[g], u, v, w)
    srv.drain()
    t1 = time.perf_counter()
    done = []
    while True:
        part = srv.poll(cap=4096)
        if not part:
            break
        done += part
    srv.close()
    return done, t1 - t0


def run_serving(args, cfg):
    """Serving form at several arrival rates: the server (coalescing, several
    workers, admission against 120 GB) against the plain per-request GPU path
    (one request per batch, one at a time), on identical graph copies."""
    import torch
    W = _module("workloads")
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    hl = importlib.import_module("hit-leiden_b200")
    graphs = W.config5(args.seed + rank, scale=args.scale)
    A = _load_many(hl, graphs, args.levels, local)
    B = _load_many(hl, graphs, args.levels, local)
    rng = np.random.default_rng(args.seed + 99)
    rates = [100.0, 1000.0, 10000.0]
    per_rate = []
    for ri, rate in enumerate(rates):
        nreq = args.requests
        gsel = rng.integers(0, len(graphs), nreq)
        sizes = np.exp(rng.uniform(np.log(10), np.log(100_000), nreq)).astype(np.int64)
        reqs = []
        for j in range(nreq):
            n, s, d, w = graphs[gsel[j]]
            u, v, ww = W.fast_batch(n, s, d, int(sizes[j]), 0.85, 17 + 1000 * ri + j)
            reqs.append((int(gsel[j]), u, v, ww))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
        res = {}
        for name, states, workers, coalesce in (("served", A, args.workers, None),
                                                ("plain", B, 1, 1)):
            done, wall = _serve(hl, states, reqs, arrivals, workers, coalesce, 120 * 10**9)
            ok = [d for d in done if d["status"] == 0]
            lat = sorted(d["latency_ms"] for d in ok)
            e = sum(d["edges"] for d in ok)
            l0 = sorted(d["level0_ms"] for d in ok)
            res[name] = {"edge_updates_per_s": e / wall, "p50_ms": lat[len(lat) // 2],
                         "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                         "level0_p50_ms": l0[len(l0) // 2],
                         "batches": len({d["batch_id"] for d in ok}), "requests": len(ok),
                         "rejected": len(done) - len(ok)}
        per_rate.append({"rate_req_s": rate, **{f"{k}_{m}": v for k, r in res.items()
                                                for m, v in r.items()}})
    top = per_rate[-1]
    if rank == 0:
        line = {
            "metric": "edge_updates_per_s", "value": top["served_edge_updates_per_s"],
            "unit": "edge-updates/s", "n_gpus": 1, "steps": len(rates), "warmup": 0,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg["workload"], "scale": args.scale, "graphs": len(graphs),
                       "vertices": int(sum(g[0] for g in graphs)),
                       "edges": int(sum(len(g[1]) for g in graphs)), "workers": args.workers,
                       "requests_per_rate": args.requests,
                       "timing": "host clock, first submit to last completion",
                       "rates": per_rate},
            "e2e": {"value": top["served_edge_updates_per_s"], "unit": "edge-updates/s",
                    "p50_ms": top["served_p50_ms"], "p99_ms": top["served_p99_ms"]},
            "roofline": None, "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    for st in A + B:
        st.close()


def _roof(kernels, key, label, peak, peak_kind):
    ev = kernels.get(key, {})
    if not ev.get("launches") or not ev.get("ms"):
        return None
    achieved = ev["bytes"] / (ev["ms"] / 1000.0) / 1e9
    return {"kernel": label, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind,
            "bytes_per_launch": ev["bytes"] / ev["launches"],
            "avg_launch_ms": ev["ms"] / ev["launches"], "traffic": None}


def _device_bytes(L, h):
    used, peak = C.c_uint64(), C.c_uint64()
    L.check(L.lib.hl_device_bytes(h, C.byref(used), C.byref(peak)))
    return {"used": used.value, "peak": peak.value}


def _pinned(batches):
    """Batches as pinned host tensors (u32 viewed as int32, f64)."""
    import torch
    out = []
    for (u, v, w) in batches:
        if isinstance(u, np.ndarray):
            tu = torch.from_numpy(np.ascontiguousarray(u).view(np.int32))
            tv = torch.from_numpy(np.ascontiguousarray(v).view(np.int32))
            tw = torch.from_numpy(np.ascontiguousarray(w))
        else:
            tu, tv, tw = u, v, w
        out.append(tuple(torch.empty(t.shape, dtype=t.dtype, pin_memory=True).copy_(t)
                         for t in (tu, tv, tw)))
    return out


def _timed_steps(L, h, pinned, n, rep, clocks):
    """The K timed steps, each through the public host API: hl_apply_batch on
    a pinned host batch (its host→device copy inside), then hl_get_map of the
    level-0 communities into pinned host memory.  A barrier and a device
    synchronise bracket the K steps.  Returns per-step device ms (CUDA events
    on the library's stream, from the batch resident in HBM), per-step host
    seconds, launches and traversed entries."""
    import torch
    comm = torch.empty(n, dtype=torch.int32, pin_memory=True)
    stats = L.BatchStats()
    dev_ms, host_s, launches, traversed = [], [], 0, 0
    clocks.start()
    rep.barrier()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("hl_timed")
    for (pu, pv, pw) in pinned:
        t1 = time.perf_counter()
        L.check(L.lib.hl_apply_batch(h, C.c_void_p(pu.data_ptr()), C.c_void_p(pv.data_ptr()),
                                     C.c_void_p(pw.data_ptr()), pu.numel(), C.byref(stats)))
        L.check(L.lib.hl_get_map(h, 0, L.HL_MAP_COMMUNITY, C.c_void_p(comm.data_ptr())))
        host_s.append(time.perf_counter() - t1)
        dev_ms.append(stats.device_ms)
        launches += stats.launches
        traversed += stats.traversed
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    rep.barrier()
    return dev_ms, host_s, launches, traversed, clocks.stop()


def _kernel_table(L, h):
    kst = (L.KernelStat * 32)()
    cnt = C.c_uint32()
    L.check(L.lib.hl_kernel_stats(h, kst, 32, C.byref(cnt)))
    return {kst[i].name.decode(): {"launches": kst[i].launches, "ms": kst[i].total_ms,
                                   "bytes": kst[i].bytes, "items": kst[i].items}
            for i in range(cnt.value)}


def _bench_line(rep, cfg_workload, config, K, Wm, k, n, dev_ms, host_s, launches, traversed,
                kernels, clk, roof_traffic):
    tot_ms = rep.max_over_ranks(float(sum(dev_ms)))
    tot_host = rep.max_over_ranks(float(sum(host_s)))
    value = rep.whole_job_rate(K, k, tot_ms / 1000.0)
    e2e_val = rep.whole_job_rate(K, k, tot_host)
    lat = sorted(1000.0 * x for x in host_s)
    dlat = sorted(dev_ms)
    peak, peak_kind = measured_peak()
    roof = _roof(kernels, "move_eval", "k_eval_* and k_pb_* <EVAL_MOVE> (inc-movement best-move "
                 "evaluation: all degree bins and the partitioned hub pass)", peak, peak_kind)
    if roof is not None and roof_traffic:
        roof["traffic"] = roof["bytes_per_launch"] * roof_traffic
    mv = kernels.get("stage_move", {})
    return {
        "metric": "edge_updates_per_s", "value": value, "unit": "edge-updates/s",
        "n_gpus": rep.world, "steps": K, "warmup": Wm, "ms_per_step": tot_ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config,
        "e2e": {"value": e2e_val, "unit": "edge-updates/s",
                "h2d_bytes_per_step": int(k * (4 + 4 + 8)), "d2h_bytes_per_step": int(n * 4),
                "p50_ms": lat[len(lat) // 2],
                "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                "note": "the same K batches as value, timed on the host clock around "
                        "hl_apply_batch (pinned host batch in) and hl_get_map (level-0 map "
                        "out into pinned memory)"},
        "device_p50_ms": dlat[len(dlat) // 2],
        "device_p99_ms": dlat[min(len(dlat) - 1, int(0.99 * len(dlat)))],
        "gpu_launches": int(launches),
        "traversed_edges_per_s": traversed / (mv["ms"] / 1000.0) if mv.get("ms") else None,
        "roofline": roof,
        "roofline_aggregation": _roof(kernels, "aggregate_compress",
                                      "inc-aggregation (emission + compression)", peak,
                                      peak_kind),
        "clocks": clk,
    }


def run_rmat(args, cfg):
    """R-MAT scale 25: graph and batches generated on the GPU (torch, input
    plumbing only), the graph loaded with hl_create_device; every step applies
    a pinned host batch through hl_apply_batch and reads the level-0 map."""
    import torch
    R = importlib.import_module("hit-leiden_b200.replicas")
    W = _module("workloads")
    rep = R.Replicas("nccl")
    local = rep.local
    torch.cuda.set_device(local)
    hl = importlib.import_module("hit-leiden_b200")
    L = importlib.import_module("hit-leiden_b200._lib")
    scale = 25 if not args.ncu_small else 20
    n, bs, bd = W.rmat_torch(scale, 16, args.seed + rep.rank, device=f"cuda:{local}")
    m = bs.numel()
    torch.cuda.empty_cache()  # hand the generator's cached blocks back before the load
    free_b, total_b = torch.cuda.mem_get_info()
    print(f"# R-MAT scale {scale}: {n} vertices, {m} edges; device free {free_b} of {total_b}",
          file=sys.stderr, flush=True)
    k = cfg["batch"] if not args.ncu_small else 1_000_000 >> 5
    rc = hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=args.levels, device=local)
    c = rc.to_c()
    c.flags |= L.HL_FLAG_KERNEL_TIMING
    h = C.c_void_p()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L.check(L.lib.hl_create_device(C.byref(c), n, C.c_void_p(bs.data_ptr()),
                                   C.c_void_p(bd.data_ptr()), None, m, C.byref(h)))
    boot_s = time.perf_counter() - t0
    st = hl.PartitionState(h, n, rc)
    q_boot = st.modularity()
    K, Wm = args.steps, args.warmup
    seeds = iter(range(10_000, 20_000))
    pinned = _pinned([W.rmat_batch_torch(scale, bs, bd, k, 0.9, next(seeds))
                      for _ in range(Wm + K)])
    # base edges the serving phase's requests delete from
    gsel = torch.Generator(device=bs.device)
    gsel.manual_seed(args.seed + 77)
    pick = torch.randint(0, bs.numel(), (1 << 21,), generator=gsel, device=bs.device)
    del_pool = (bs[pick].cpu().numpy().view(np.uint32), bd[pick].cpu().numpy().view(np.uint32))
    del bs, bd, pick
    torch.cuda.empty_cache()
    for (pu, pv, pw) in pinned[:Wm]:
        L.check(L.lib.hl_apply_batch(h, C.c_void_p(pu.data_ptr()), C.c_void_p(pv.data_ptr()),
                                     C.c_void_p(pw.data_ptr()), k, None))
    torch.cuda.synchronize()
    L.check(L.lib.hl_reset_kernel_stats(h))
    dev_ms, host_s, launches, traversed, clk = _timed_steps(L, h, pinned[Wm:], n, rep,
                                                           Clocks(local))
    kernels = _kernel_table(L, h)
    # the committed ratio is measured at scale 25; the small case has none
    tr = None if args.ncu_small else committed_traffic(args.config)
    ratio = (tr or {}).get("traffic_per_algorithmic_byte")
    config = {"workload": cfg["workload"], "scale": scale, "vertices": n, "edges": int(m),
              "batch_edges": k, "levels": st.levels, "parallelism": f"replicas{rep.world}",
              "l2": "inputs larger than L2 (resident CSR > 126 MB); no flush",
              "bootstrap_s": boot_s, "bootstrap_modularity": q_boot}
    line = _bench_line(rep, cfg["workload"], config, K, Wm, k, n, dev_ms, host_s, launches,
                       traversed, kernels, clk, ratio)
    q = st.modularity()
    dbytes = _device_bytes(L, h)
    tmid, twide, tdef, tfr = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    L.check(L.lib.hl_autotune_info(h, C.byref(tmid), C.byref(twide), C.byref(tdef),
                                   C.byref(tfr)))
    config["degree_bins"] = {"warp_table_max": tmid.value, "wide_max": twide.value,
                             "hub_defer_entries": tdef.value, "tuned_on_frontier": tfr.value}
    served = None
    if not args.no_served:
        served = _served_rmat(hl, st, scale, del_pool, args.seed, torch, args.served_requests)
    st.close()
    cpu = None
    if rep.rank == 0 and rep.world == 1 and not args.no_cpu_baseline:
        r = cpu_rmat_sample(args.seed, args.levels, 0, args.cpu_sample_batches,
                            args.cpu_sample_cap, args.rmat_sample_scale)
        cpu = {"value": r["value"], "unit": "edge-updates/s", "cores": r["threads"],
               "kind": "port", "sample": _rmat_sample_text(r)}
    if rep.rank == 0:
        line.update({"cpu_baseline": cpu, "modularity": q, "kernels": kernels,
                     "device_bytes": dbytes, "served": served})
        print(json.dumps(line), flush=True)
    rep.close()


def _served_rmat(hl, st, scale, del_pool, seed, torch, requests):
    """The serving form on the resident R-MAT graph: `requests` edge-update
    requests (sizes log-uniform in [10, 100k], 85% R-MAT inserts / 15% deletes)
    arrive as a Poisson stream at 10,000 requests/s; the server coalesces the
    ones that arrive while the graph is busy.  Against it, the plain
    per-request path applies a few requests of the same stream one per batch.
    Host clock; requests from host memory."""
    rng = np.random.default_rng(seed + 123)
    sizes = np.exp(rng.uniform(np.log(10), np.log(100_000), requests)).astype(np.int64)
    eu, ev = del_pool  # base edges (deleting one that is already gone is a no-op)

    def request(j, sz):
        g = np.random.default_rng(seed * 7919 + j)
        ki = int(round(sz * 0.85))
        kd = int(sz) - ki
        u = np.zeros(ki, np.int64)
        v = np.zeros(ki, np.int64)
        for lvl in range(scale):
            r = g.random(ki)
            u |= (r >= 0.76).astype(np.int64) << lvl
            v |= (((r >= 0.57) & (r < 0.76)) | (r >= 0.95)).astype(np.int64) << lvl
        keep = u != v
        u, v = u[keep], v[keep]
        di = g.integers(0, len(eu), kd)
        uu = np.concatenate([np.minimum(u, v), eu[di]]).astype(np.uint32)
        vv = np.concatenate([np.maximum(u, v), ev[di]]).astype(np.uint32)
        ww = np.concatenate([np.ones(len(u)), -np.ones(kd)])
        return uu, vv, ww
    reqs = [request(j, sz) for j, sz in enumerate(sizes)]
    plain_reqs = [request(10_000 + j, sz) for j, sz in enumerate(sizes[:3])]
    arrivals = np.cumsum(rng.exponential(1.0 / 10_000.0, requests))
    torch.cuda.synchronize()
    level_events = []
    srv = hl.Server(workers=1)
    srv.set_level_callback(lambda graph, batch, level, nodes, ids:
                           level_events.append((batch, level, len(nodes))))
    gid = srv.add(st)
    t0 = time.perf_counter()
    for (u, v, w), ta in zip(reqs, arrivals):
        while time.perf_counter() - t0 < ta:
            pass
        srv.submit(gid, u, v, w)
    srv.drain()
    wall = time.perf_counter() - t0
    done = []
    while True:
        part = srv.poll(cap=4096)
        if not part:
            break
        done += part
    srv.close()
    ok = [d for d in done if d["status"] == 0]
    edges = sum(d["edges"] for d in ok)
    lat = sorted(d["latency_ms"] for d in ok)
    l0 = sorted(d["level0_ms"] for d in ok)
    # plain per-request path: one request per batch, same stream
    tp = 0.0
    ep = 0
    for (u, v, w) in plain_reqs:
        t1 = time.perf_counter()
        st.apply_batch(u, v, w)
        tp += time.perf_counter() - t1
        ep += len(u)
    served_rate = edges / wall
    plain_rate = ep / tp
    return {"requests": len(ok), "rejected": len(done) - len(ok), "edges": int(edges),
            "batches": len({d["batch_id"] for d in ok}), "arrival_rate_req_s": 10_000,
            "edge_updates_per_s": served_rate, "p50_ms": lat[len(lat) // 2],
            "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
            "level0_p50_ms": l0[len(l0) // 2],
            "plain_per_request_edge_updates_per_s": plain_rate,
            "plain_requests_timed": len(plain_reqs),
            "served_over_plain": served_rate / plain_rate,
            "timing": "host clock: first submit to last completion (served); the plain "
                      "requests one per hl_apply_batch"}


def main():
    args = parse()
    cfg = CONFIGS[args.config]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.cpu_variant_run:
        return run_cpu_variant(args)
    if args.impl == "reference":
        # the CPU port on the host cores: rank 0 alone works under torchrun
        if rank == 0:
            if args.config in ("batch256", "serve32"):
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference updates one PartitionState per call and has no "
                                  "batching or serving form; its per-graph path is the rmat25 / "
                                  "lfr1m / ca_hepth reference arm"}), flush=True)
            else:
                run_reference(args, cfg)
        return
    if args.config == "rmat25":
        return run_rmat(args, cfg)
    if args.config == "batch256":
        return run_batching(args, cfg)
    if args.config == "serve32":
        return run_serving(args, cfg)
    import torch
    R = importlib.import_module("hit-leiden_b200.replicas")
    rep = R.Replicas("nccl")
    torch.cuda.set_device(local)
    hl = importlib.import_module("hit-leiden_b200")
    L = importlib.import_module("hit-leiden_b200._lib")

    n, s, d, w, wts, ins, pref = make_graph(args.config, args.seed, args.ncu_small)
    k = cfg["batch"]
    K, Wm = args.steps, args.warmup
    n_cpu = 0 if (args.no_cpu_baseline or rank != 0 or world != 1) else args.cpu_sample_batches
    batches = make_batches(n, s, d, w, wts, ins, pref, Wm + K + n_cpu, k, args.seed)

    rc = hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=args.levels, device=local)
    c = rc.to_c()
    c.flags |= L.HL_FLAG_KERNEL_TIMING
    h = C.c_void_p()
    t0 = time.perf_counter()
    L.check(L.lib.hl_create(C.byref(c), n, L.ptr(s), L.ptr(d), L.ptr(w), len(s), C.byref(h)))
    boot_s = time.perf_counter() - t0
    st = hl.PartitionState(h, n, rc)
    for (u, v, ww) in batches[:Wm]:
        st.apply_batch(u, v, ww)
    pinned = _pinned(batches[Wm:Wm + K])
    torch.cuda.synchronize()
    L.check(L.lib.hl_reset_kernel_stats(h))
    dev_ms, host_s, launches, traversed, clk = _timed_steps(L, h, pinned, n, rep, Clocks(local))
    kernels = _kernel_table(L, h)
    tr = None if args.ncu_small else committed_traffic(args.config)
    ratio = (tr or {}).get("traffic_per_algorithmic_byte")
    config = {"workload": cfg["workload"], "vertices": n, "edges": int(len(s)),
              "batch_edges": k, "levels": st.levels, "parallelism": f"replicas{world}",
              "l2": "inputs larger than L2 (resident CSR > 126 MB); no flush",
              "bootstrap_s": boot_s}
    line = _bench_line(rep, cfg["workload"], config, K, Wm, k, n, dev_ms, host_s, launches,
                       traversed, kernels, clk, ratio)
    q = st.modularity()
    cpu = None
    if n_cpu:
        r = cpu_baseline(st, batches[Wm + K:], n_cpu, args.cpu_sample_cap)
        cpu = {"value": r["value"], "unit": "edge-updates/s", "cores": r["threads"],
               "kind": "port",
               "sample": f"{r['batches']} batch(es) of {k} updates of the same stream, right "
                         f"after the timed ones, from the GPU's state (median "
                         f"{statistics.median(r['batch_s']):.2f} s a batch on {r['threads']} "
                         "host threads)",
               "parity_bit_exact_after_sample": r["parity_bit_exact"],
               "dq_after_sample": r["dq"]}
    if rank == 0:
        line.update({"cpu_baseline": cpu, "modularity": q, "kernels": kernels})
        print(json.dumps(line), flush=True)
    st.close()
    rep.close()


if __name__ == "__main__":
    main()
