#!/usr/bin/env python3
"""Benchmark of the HIT-Leiden incremental update path on B200.

One step = one edge-update batch applied through hl_apply_batch (G ⊕ ΔG, then
inc-movement, inc-refinement and inc-aggregation on every level, then the
top-down level maps), on a graph already resident in HBM.

Default workload (the mid-size plain-method configuration): LFR-style planted
graph, 1M vertices / ~20M undirected edges, degree exponent 2.5 (mean 40, max
2000), community sizes exponent 1.5 in [50, 5000], mixing 0.3, f64 weights
U[0.5, 2.0]; batches of 10k updates (90% degree-preferential inserts, 10%
uniform deletes of existing edges).  Synthetic, seeded: the reference's
datasets are not available.

Reported:
  value   edge-updates/s with batches already on the device (hl_apply_batch_device),
          timed by CUDA events on the library's stream, summed over the K steps;
  e2e     edge-updates/s through the public host API (hl_apply_batch with
          batches in pinned host memory, host→device copies inside) plus a
          device→host read of the level-0 community map into pinned memory
          every step, timed on the host clock;
  roofline for the inc-movement evaluation kernel (algorithmic bytes / event time);
  cpu_baseline: the CPU oracle (a C++ port of the reference's Rust, its
          snapshot evaluations on all host threads as the reference's rayon
          pool) applying one batch of the same stream from the same state.

--impl reference runs that CPU port alone on the same configuration.
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
    ap.add_argument("--config", choices=sorted(CONFIGS), default="lfr1m")
    ap.add_argument("--levels", type=int, default=10)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-sample-batches", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-variants", action="store_true",
                    help="reference arm: also time the faithful CPU variants (the "
                         "reference's quadratic refinement scans; throughput on all host "
                         "threads and deterministic on one) and a from-scratch run() on "
                         "the updated graph, one batch each under --cpu-cap")
    ap.add_argument("--cpu-cap", type=float, default=120.0,
                    help="wall-clock cap in seconds for each faithful variant's batch")
    ap.add_argument("--cpu-variant-run", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-variant-mode", default="throughput", help=argparse.SUPPRESS)
    ap.add_argument("--ncu-small", action="store_true",
                    help="small case for ncu captures (200k vertices)")
    ap.add_argument("--workers", type=int, default=16,
                    help="host worker threads of the batching / serving forms")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="vertex-count scale of the serving form's graphs")
    ap.add_argument("--requests", type=int, default=400,
                    help="requests per arrival rate in the serving form")
    return ap.parse_args()


def make_graph(cfg_name, seed, small=False):
    W = importlib.import_module("hit-leiden_b200.workloads")
    if cfg_name == "lfr1m":
        if small:
            n, s, d, w = W.config2(seed, n=200_000)
        else:
            n, s, d, w = W.config2(seed)
        return n, s, d, w, (0.5, 2.0), 0.9, True
    n, s, d, w = W.config1(seed)
    return n, s, d, w, None, 1.0, False


def make_batches(n, s, d, w, weights, insert_frac, preferential, count, k, seed):
    W = importlib.import_module("hit-leiden_b200.workloads")
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


def committed_traffic():
    """Per-launch DRAM bytes of the evaluation kernel from the committed ncu
    summary, scaled to the bench's launch (see profiles/)."""
    p = os.path.join(ROOT, "profiles", "move_eval_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
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


def cpu_baseline(st, batches, levels_cfg, max_batches):
    """Time the oracle port on the next batches from the GPU's state; check that
    the GPU state after the same batches is identical (full-size parity)."""
    from oracle import oracle as O
    O.load()
    ora = O.State(st.node_count, levels=1, mode=O.MODE_THROUGHPUT)
    ora.import_levels(export_state(st))
    t_cpu = 0.0
    edges = 0
    used = 0
    for (u, v, w) in batches[:max_batches]:
        t0 = time.perf_counter()
        ora.hit_leiden(u, v, w)
        t_cpu += time.perf_counter() - t0
        edges += len(u)
        used += 1
        st.apply_batch(u, v, w)
    same = st.levels == ora.levels and all(
        np.array_equal(st.community_mapping_per_level[p], ora.get_map(p, O.MAP_F))
        and np.array_equal(st.current_subcommunity_mapping_per_level[p],
                           ora.get_map(p, O.MAP_S_CUR))
        for p in range(ora.levels))
    q_gpu = st.modularity()
    q_cpu = ora.modularity(0)
    return {"value": edges / t_cpu, "seconds": t_cpu, "batches": used, "edges": edges,
            "parity_bit_exact": bool(same), "dq": abs(q_gpu - q_cpu),
            "threads": O.num_threads()}


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
    """CPU port of the reference path alone (bootstrap untimed, then K batches)."""
    from oracle import oracle as O
    O.load()
    n, s, d, w, wts, ins, pref = make_graph(args.config, args.seed, args.ncu_small)
    k = cfg["batch"]
    steps = max(1, min(args.steps, 2))
    warm = 0
    batches = make_batches(n, s, d, w, wts, ins, pref, warm + steps, k, args.seed)
    st = O.State(n, mode=O.MODE_THROUGHPUT)
    if args.levels > 1:
        st.bootstrap(s, d, w, max_levels=args.levels)
    else:
        st = O.State(n, levels=1, mode=O.MODE_THROUGHPUT)
        st.push_empty_graph()
        st.hit_leiden(s, d, w)
    variants = _time_variants(st, batches[warm], k, args.cpu_cap) if args.cpu_variants else None
    t = 0.0
    q_first = None
    for (u, v, ww) in batches[warm:]:
        t0 = time.perf_counter()
        st.hit_leiden(u, v, ww)
        t += time.perf_counter() - t0
        if variants is not None and q_first is None:
            q_first = st.modularity(0)
    val = steps * k / t
    if variants and "modularity" in variants["faithful_throughput"]:
        # the faithful scans change the cost, not the result
        variants["faithful_throughput"]["same_result"] = (
            variants["faithful_throughput"]["modularity"] == q_first)
    line = {
        "impl": "reference", "metric": "edge_updates_per_s", "value": val,
        "unit": "edge-updates/s", "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * t / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": cfg["workload"], "levels": st.levels, "batch_edges": k},
        "cpu_baseline": {"value": val, "unit": "edge-updates/s", "cores": O.num_threads(),
                         "kind": "port",
                         "sample": f"{steps} batches of {k} updates after an untimed bootstrap "
                                   "(snapshot evaluations on all host threads, up to 64)"},
        "e2e": {"value": val, "unit": "edge-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "modularity": st.modularity(0),
    }
    if variants is not None:
        line["cpu_variants"] = variants
    print(json.dumps(line), flush=True)


def _load_many(hl, graphs, levels, device, threads=16):
    """Load and bootstrap many graphs concurrently (each on its own stream)."""
    from concurrent.futures import ThreadPoolExecutor

    def one(g):
        n, s, d, w = g
        return hl.PartitionState.load(hl.GraphInput.from_arrays("g", n, s, d, w),
                                      hl.RunConfig(max_iterations=levels, device=device))
    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(one, graphs))


def run_batching(args, cfg):
    """Batching form: every step applies one batch to each of 256 graphs, once
    through hl_apply_batches (graphs concurrent) and once through the plain
    per-graph path (a loop of hl_apply_batch) on an identical copy; both from
    host arrays, host clock with the device synchronised on both sides."""
    import torch
    R = importlib.import_module("hit-leiden_b200.replicas")
    W = importlib.import_module("hit-leiden_b200.workloads")
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
    W = importlib.import_module("hit-leiden_b200.workloads")
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
            res[name] = {"edge_updates_per_s": e / wall, "p50_ms": lat[len(lat) // 2],
                         "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
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


def run_rmat(args, cfg):
    """R-MAT scale 25: graph and batches generated on the GPU (torch, input
    plumbing only), loaded with hl_create_device; value from device-resident
    batches (CUDA events), e2e through hl_apply_batch with host arrays."""
    import torch
    R = importlib.import_module("hit-leiden_b200.replicas")
    W = importlib.import_module("hit-leiden_b200.workloads")
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
    k = cfg["batch"] if not args.ncu_small else 50_000
    rc = hl.RunConfig(max_iterations=args.levels, device=local)
    c = rc.to_c()
    c.flags |= L.HL_FLAG_KERNEL_TIMING
    h = C.c_void_p()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L.check(L.lib.hl_create_device(C.byref(c), n, C.c_void_p(bs.data_ptr()),
                                   C.c_void_p(bd.data_ptr()), None, m, C.byref(h)))
    boot_s = time.perf_counter() - t0
    st = hl.PartitionState(h, n, rc)
    K, Wm = args.steps, args.warmup
    seeds = iter(range(10_000, 20_000))
    for _ in range(Wm):
        u, v, w = W.rmat_batch_torch(scale, bs, bd, k, 0.9, next(seeds))
        L.check(L.lib.hl_apply_batch_device(h, C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()),
                                            C.c_void_p(w.data_ptr()), k, None))
    dev = [W.rmat_batch_torch(scale, bs, bd, k, 0.9, next(seeds)) for _ in range(K)]
    torch.cuda.synchronize()
    L.check(L.lib.hl_reset_kernel_stats(h))
    clocks = Clocks(local)
    clocks.start()
    rep.barrier()
    torch.cuda.synchronize()
    dev_ms, launches, traversed = [], 0, 0
    stats = L.BatchStats()
    torch.cuda.nvtx.range_push("hl_timed")
    for (u, v, w) in dev:
        L.check(L.lib.hl_apply_batch_device(h, C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()),
                                            C.c_void_p(w.data_ptr()), k, C.byref(stats)))
        dev_ms.append(stats.device_ms)
        launches += stats.launches
        traversed += stats.traversed
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    rep.barrier()
    clk = clocks.stop()
    tot_ms = rep.max_over_ranks(float(sum(dev_ms)))
    value = rep.whole_job_rate(K, k, tot_ms / 1000.0)
    kst = (L.KernelStat * 32)()
    cnt = C.c_uint32()
    L.check(L.lib.hl_kernel_stats(h, kst, 32, C.byref(cnt)))
    kernels = {kst[i].name.decode(): {"launches": kst[i].launches, "ms": kst[i].total_ms,
                                      "bytes": kst[i].bytes, "items": kst[i].items}
               for i in range(cnt.value)}
    del dev
    # end to end: host arrays in, level-0 map out
    host = []
    for _ in range(K):
        u, v, w = W.rmat_batch_torch(scale, bs, bd, k, 0.9, next(seeds))
        host.append((u.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32),
                     w.cpu().numpy()))
    comm = np.zeros(n, np.uint32)
    rep.barrier()
    torch.cuda.synchronize()
    e2e_s = []
    for (u, v, w) in host:
        t1 = time.perf_counter()
        st.apply_batch(u, v, w)
        L.check(L.lib.hl_get_map(h, 0, L.HL_MAP_COMMUNITY, L.ptr(comm)))
        e2e_s.append(time.perf_counter() - t1)
    tot_e2e = rep.max_over_ranks(float(sum(e2e_s)))
    e2e_val = rep.whole_job_rate(K, k, tot_e2e)
    lat = sorted(1000.0 * x for x in e2e_s)
    peak, peak_kind = measured_peak()
    mv = kernels.get("stage_move", {})
    if rep.rank == 0:
        line = {
            "metric": "edge_updates_per_s", "value": value, "unit": "edge-updates/s",
            "n_gpus": rep.world, "steps": K, "warmup": Wm, "ms_per_step": tot_ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": cfg["workload"], "scale": scale, "vertices": n,
                       "edges": int(m), "batch_edges": k, "levels": st.levels,
                       "parallelism": f"replicas{rep.world}",
                       "l2": "inputs larger than L2 (resident CSR > 126 MB)",
                       "bootstrap_s": boot_s},
            "e2e": {"value": e2e_val, "unit": "edge-updates/s",
                    "h2d_bytes_per_step": int(k * 16), "d2h_bytes_per_step": int(n * 4),
                    "p50_ms": lat[len(lat) // 2],
                    "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
            "gpu_launches": int(launches),
            "traversed_edges_per_s": traversed / (mv["ms"] / 1000.0) if mv.get("ms") else None,
            "roofline": _roof(kernels, "move_eval",
                              "k_eval<EVAL_MOVE> (inc-movement best-move evaluation)", peak,
                              peak_kind),
            "roofline_aggregation": _roof(kernels, "aggregate_compress",
                                          "inc-aggregation (emission + compression)", peak,
                                          peak_kind),
            "cpu_baseline": None,
            "cpu_baseline_note": "the CPU port is not run at 500M edges (a single batch "
                                 "would take hours on one core)",
            "clocks": clk, "modularity": st.modularity(), "kernels": kernels,
            "device_bytes": _device_bytes(L, h),
        }
        print(json.dumps(line), flush=True)
    st.close()
    rep.close()


def main():
    args = parse()
    cfg = CONFIGS[args.config]
    if args.impl == "ours" and args.config == "rmat25":
        return run_rmat(args, cfg)
    if args.impl == "ours" and args.config == "batch256":
        return run_batching(args, cfg)
    if args.impl == "ours" and args.config == "serve32":
        return run_serving(args, cfg)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.cpu_variant_run:
        return run_cpu_variant(args)
    if args.impl == "reference":
        if rank == 0:
            if args.config in ("batch256", "serve32", "rmat25"):
                print(json.dumps({"impl": "reference", "unavailable":
                                  "not run for this configuration: the CPU port's per-graph "
                                  "path is the lfr1m / ca_hepth reference arm"}), flush=True)
            else:
                run_reference(args, cfg)
        return
    import torch
    R = importlib.import_module("hit-leiden_b200.replicas")
    rep = R.Replicas("nccl")
    torch.cuda.set_device(local)
    hl = importlib.import_module("hit-leiden_b200")
    L = importlib.import_module("hit-leiden_b200._lib")
    barrier = rep.barrier

    n, s, d, w, wts, ins, pref = make_graph(args.config, args.seed, args.ncu_small)
    k = cfg["batch"]
    K, Wm = args.steps, args.warmup
    n_cpu = 0 if (args.no_cpu_baseline or rank != 0 or world != 1) else args.cpu_sample_batches
    batches = make_batches(n, s, d, w, wts, ins, pref, Wm + 2 * K + n_cpu, k, args.seed)

    rc = hl.RunConfig(max_iterations=args.levels, device=local)
    c = rc.to_c()
    c.flags |= L.HL_FLAG_KERNEL_TIMING
    h = C.c_void_p()
    t0 = time.perf_counter()
    L.check(L.lib.hl_create(C.byref(c), n, L.ptr(s), L.ptr(d), L.ptr(w), len(s), C.byref(h)))
    boot_s = time.perf_counter() - t0
    st = hl.PartitionState(h, n, rc)

    for (u, v, ww) in batches[:Wm]:
        st.apply_batch(u, v, ww)

    # device-resident batches for the HBM-resident measurement
    dev = []
    for (u, v, ww) in batches[Wm:Wm + K]:
        dev.append((torch.from_numpy(u.view(np.int32)).to(f"cuda:{local}"),
                    torch.from_numpy(v.view(np.int32)).to(f"cuda:{local}"),
                    torch.from_numpy(ww).to(f"cuda:{local}")))
    torch.cuda.synchronize()
    L.check(L.lib.hl_reset_kernel_stats(h))
    clocks = Clocks(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    dev_ms = []
    launches = 0
    traversed = 0
    stats = L.BatchStats()
    torch.cuda.nvtx.range_push("hl_timed")
    for (du, dv, dw) in dev:
        L.check(L.lib.hl_apply_batch_device(h, C.c_void_p(du.data_ptr()), C.c_void_p(dv.data_ptr()),
                                            C.c_void_p(dw.data_ptr()), k, C.byref(stats)))
        dev_ms.append(stats.device_ms)
        launches += stats.launches
        traversed += stats.traversed
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    tot_ms = rep.max_over_ranks(float(sum(dev_ms)))
    value = rep.whole_job_rate(K, k, tot_ms / 1000.0)

    kst = (L.KernelStat * 32)()
    cnt = C.c_uint32()
    L.check(L.lib.hl_kernel_stats(h, kst, 32, C.byref(cnt)))
    kernels = {kst[i].name.decode(): {"launches": kst[i].launches, "ms": kst[i].total_ms,
                                      "bytes": kst[i].bytes, "items": kst[i].items}
               for i in range(cnt.value)}

    # end to end through the host API: each batch is copied in from pinned host
    # memory and the level-0 community map read back into pinned host memory
    e2e_s = []
    pinned = [(torch.from_numpy(u.view(np.int32)).pin_memory(),
               torch.from_numpy(v.view(np.int32)).pin_memory(),
               torch.from_numpy(ww).pin_memory()) for (u, v, ww) in batches[Wm + K:Wm + 2 * K]]
    comm = torch.empty(n, dtype=torch.int32).pin_memory()
    e2e_stats = L.BatchStats()
    barrier()
    torch.cuda.synchronize()
    for (pu, pv, pw) in pinned:
        t1 = time.perf_counter()
        L.check(L.lib.hl_apply_batch(h, C.c_void_p(pu.data_ptr()), C.c_void_p(pv.data_ptr()),
                                     C.c_void_p(pw.data_ptr()), pu.numel(),
                                     C.byref(e2e_stats)))
        L.check(L.lib.hl_get_map(h, 0, L.HL_MAP_COMMUNITY, C.c_void_p(comm.data_ptr())))
        e2e_s.append(time.perf_counter() - t1)
    torch.cuda.synchronize()
    barrier()
    tot_e2e = rep.max_over_ranks(float(sum(e2e_s)))
    e2e_val = rep.whole_job_rate(K, k, tot_e2e)
    lat = sorted(1000.0 * x for x in e2e_s)

    ev = kernels.get("move_eval", {})
    peak, peak_kind = measured_peak()
    roof = None
    if ev.get("launches"):
        achieved = ev["bytes"] / (ev["ms"] / 1000.0) / 1e9
        per_launch = ev["bytes"] / ev["launches"]
        tr = committed_traffic()
        traffic = None
        if tr and tr.get("config") == args.config and tr.get("traffic_per_algorithmic_byte"):
            traffic = per_launch * tr["traffic_per_algorithmic_byte"]
        roof = {"kernel": "k_eval<EVAL_MOVE> (inc-movement best-move evaluation)",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "bytes_per_launch": per_launch, "avg_launch_ms": ev["ms"] / ev["launches"],
                "traffic": traffic}

    q = st.modularity()
    cpu = None
    if n_cpu:
        cpu_res = cpu_baseline(st, batches[Wm + 2 * K:], args.levels, n_cpu)
        cpu = {"value": cpu_res["value"], "unit": "edge-updates/s", "cores": cpu_res["threads"],
               "kind": "port",
               "sample": f"{cpu_res['batches']} batch(es) of {k} updates of the same stream, "
                         f"from the GPU's state ({cpu_res['seconds']:.1f} s on "
                         f"{cpu_res['threads']} host threads)",
               "parity_bit_exact_after_sample": cpu_res["parity_bit_exact"],
               "dq_after_sample": cpu_res["dq"]}

    if rank == 0:
        line = {
            "metric": "edge_updates_per_s", "value": value, "unit": "edge-updates/s",
            "n_gpus": world, "steps": K, "warmup": Wm, "ms_per_step": tot_ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": cfg["workload"], "vertices": n, "edges": int(len(s)),
                       "batch_edges": k, "levels": st.levels, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (resident CSR > 126 MB)",
                       "bootstrap_s": boot_s},
            "e2e": {"value": e2e_val, "unit": "edge-updates/s",
                    "h2d_bytes_per_step": int(k * (4 + 4 + 8)),
                    "d2h_bytes_per_step": int(n * 4),
                    "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1,
                                                                    int(0.99 * len(lat)))]},
            "gpu_launches": int(launches),
            "traversed_edges_per_s": (traversed / (kernels["stage_move"]["ms"] / 1000.0)
                                      if kernels.get("stage_move", {}).get("ms") else None),
            "roofline": roof,
            "roofline_aggregation": _roof(kernels, "aggregate_compress",
                                          "inc-aggregation (emission + compression)", peak,
                                          peak_kind),
            "cpu_baseline": cpu,
            "clocks": clk,
            "modularity": q,
            "kernels": kernels,
        }
        print(json.dumps(line), flush=True)
    st.close()
    rep.close()


if __name__ == "__main__":
    main()
