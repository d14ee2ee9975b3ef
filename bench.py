"""Benchmark of the B200 CSR hot path on RMAT scale 22 (edge factor 16,
uint32 ids, float32 weights in [1,256), seeded synthetic data).

A timed step is one sweep of direction-optimized BFS from 64 seeded random
roots with out-degree > 0, each search timed on the device (CUDA events),
with L2 flushed between searches.  value = Graph500 GTEPS of the sweep (sum of
out-degrees of reached vertices over search time), summed over ranks.

Also measured on the same resident graph, outside the step loop: the GPU
radix sort + CSR build (both directions, weighted), PageRank pull and push to
1e-6 L1 (max 100 iterations: iteration GTEPS and time-to-tolerance).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank owns one GPU and its own 64 roots (independent
units: weak scaling); rank 0 prints one JSON line.  --impl reference times the
reference's own OpenMP BFS (built from its sources into oracle/_ref) on the
host cores on a bounded sample of the same roots.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE, EDGE_FACTOR, SEED, NROOTS = 22, 16, 0, 64
PR_TOL, PR_MAX = 1e-6, 100
METRIC = "BFS & PR-iteration GTEPS on 1 B200 (%HBM roofline); PR time-to-1e-6, learned vs plain"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_roots(outdeg, rank: int, n: int = NROOTS) -> list[int]:
    """A rank's replica units: n distinct seeded roots with out-degree > 0
    (seed 1000 + rank, so ranks search different roots)."""
    rng = np.random.default_rng(1000 + rank)
    cand = np.nonzero(np.asarray(outdeg) > 0)[0]
    return [int(x) for x in rng.choice(cand, size=min(n, len(cand)), replace=False)]


def workload_config(ws: int) -> dict:
    """The benchmarked workload (the same for both arms)."""
    V, E = 1 << SCALE, (1 << SCALE) * EDGE_FACTOR
    return {"workload": f"RMAT scale {SCALE} (V={V}, E={E}), a/b/c/d=.57/.19/.19/.05, permuted ids, float32 weights; "
                        f"DO-BFS from {NROOTS} seeded random roots with out-degree>0 per rank, each search timed "
                        "individually",
            "global_batch": NROOTS * ws, "seq_len": None, "parallelism": f"replicas{ws}",
            "l2": "flushed (256 MB write) before every search",
            "step": f"{NROOTS} DO-BFS searches"}


def sort_passes(V: int) -> int:
    """Radix passes of the CSR build's byte model: ceil(ceil(log2 V) / 8)."""
    return -(-max(1, (V - 1).bit_length()) // 8)


def job_totals(my_ms: float, my_edges: float, ws: int, dist=None, device=None) -> tuple[float, float]:
    """Whole-job aggregate of the replicas: the slowest rank's timed
    milliseconds (max over ranks) and the edges all ranks traversed (sum)."""
    if ws == 1:
        return float(my_ms), float(my_edges)
    import torch
    t = torch.tensor([float(my_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e = torch.tensor([float(my_edges)], dtype=torch.float64, device=device)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), float(e.item())


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 25 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        """Starts sampling every 25 ms and returns once the sampler is running
        (its first line has arrived), so the timed region that follows is
        covered from its start."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "25"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10:
                time.sleep(0.005)
            self.lines.clear()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        # a region shorter than the interval still gets the sample that
        # follows it
        t0 = time.time()
        while not self.lines and time.time() - t0 < 1:
            time.sleep(0.005)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def bfs_bytes(trace, V: int) -> tuple[float, dict]:
    """Algorithmic bytes of one search from its level trace.
    TD level: 12|F| + 8 E_F + 12|N|;  BU level: 4V + 8U + 4 E_scan + 12|N|
    (U = unvisited vertices entering the level; bitmap probes cached)."""
    total, per_dir = 0.0, {"td": 0.0, "bu": 0.0}
    visited = 1
    for L in trace:
        if L["direction"] == 0:
            b = 12 * L["frontier"] + 8 * L["edges"] + 12 * L["discovered"]
            per_dir["td"] += b
        else:
            U = V - visited
            b = 4 * V + 8 * U + 4 * L["edges"] + 12 * L["discovered"]
            per_dir["bu"] += b
        total += b
        visited += L["discovered"]
    return total, per_dir


def profiled_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` (dram__bytes_read.sum +
    dram__bytes_write.sum) from its committed ncu summary, a line
    `dram_bytes_per_launch: N` in profiles/<kernel>_*.md; None if absent."""
    import glob
    for f in sorted(glob.glob(os.path.join(ROOT, "profiles", f"{kernel}_*.md"))):
        for line in open(f):
            if line.strip().startswith("dram_bytes_per_launch:"):
                try:
                    return int(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


def run_ours(args):
    import torch
    import torch.distributed as dist

    import opengraph_b200 as og

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib = og.load(True)  # the weighted layout: configs carry float32 weights
    lib.quiet(True)
    hbm_peak, peak_kind = peaks()

    # ---- inputs: RMAT-22, resident in HBM --------------------------------
    s, d, w = og.generate_rmat(SCALE, EDGE_FACTOR, SEED, weighted=True)
    V = 1 << SCALE
    E = len(s)
    ts = torch.from_numpy(s.view(np.int32)).to(dev)
    td = torch.from_numpy(d.view(np.int32)).to(dev)
    tw = torch.from_numpy(w).to(dev)
    g = lib.device_graph()
    g.build(ts, td, V, 0, weight=tw)
    torch.cuda.synchronize()
    f = g.view(False)
    outdeg = f.out_degree.cpu().numpy().view(np.uint32)
    roots = rank_roots(outdeg, rank)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    par = torch.empty(V, dtype=torch.int32, device=dev)
    dis = torch.empty(V, dtype=torch.int32, device=dev)

    def sweep():
        tot_ms, tot_edges, launches = 0.0, 0, 0
        traces = []
        for r in roots:
            flush.zero_()
            torch.cuda.synchronize()
            info = g.bfs(r, par, dis, mode=2)
            tot_ms += info["ms"]
            tot_edges += info["reached_out_edges"]
            launches += info["launches"]
            traces.append(g.bfs_trace())
        return tot_ms, tot_edges, launches, traces

    for _ in range(args.warmup):
        sweep()
    clocks = ClockSampler(local)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_ms, edges_total, launches_total, traces = [], 0, 0, None
    for _ in range(args.steps):
        ms, ed, la, traces = sweep()
        step_ms.append(ms)
        edges_total += ed
        launches_total += la
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clk = clocks.stop()
    max_ms, all_edges = job_totals(sum(step_ms), edges_total, ws, dist, dev)
    gteps = all_edges / (max_ms / 1e3) / 1e9

    # ---- roofline of the dominant kernel: bfsk_search, one launch = one search
    bu_bytes = bu_ms = td_bytes = td_ms = 0.0
    for tr in traces:
        _, per = bfs_bytes(tr, V)
        bu_bytes += per["bu"]
        td_bytes += per["td"]
        bu_ms += sum(L["ms"] for L in tr if L["direction"] == 1)
        td_ms += sum(L["ms"] for L in tr if L["direction"] == 0)
    all_bytes = sum(bfs_bytes(tr, V)[0] for tr in traces)
    sweep_ms = step_ms[-1]
    search_gbs = all_bytes / (sweep_ms / 1e3) / 1e9 if sweep_ms else 0.0
    traffic = profiled_traffic("bfsk_search")

    # ---- e2e: the reference-facing C-ABI call with host buffers ----------
    e2e = e2e_dropin(lib, og, s, d, w, roots, rank, dev)

    extra = {}
    if rank == 0 and not args.skip_stages:
        extra = stages(lib, og, g, ts, td, tw, V, E, dev, hbm_peak)

    if rank == 0 and not args.skip_stages:
        extra["batching"] = batching(lib, og, g, roots, V, E, dev, sum(step_ms) / len(step_ms), extra)
        extra["learned"] = learned_vs_plain(lib, og, g, roots, V, dev, flush, par, dis)

    cpu = None
    if rank == 0 and ws == 1 and not args.skip_cpu:
        cpu = cpu_baseline(og, s, d, w, roots[:args.cpu_roots])

    g.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC,
        "value": round(gteps, 3),
        "unit": "GTEPS",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(max_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded RMAT generator)",
        "config": workload_config(ws),
        "roofline": {"bound": "hbm", "kernel": "bfsk_search (one DO-BFS search per launch)",
                     "achieved": round(search_gbs, 1), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(search_gbs / hbm_peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic,
                     "algorithmic_bytes_per_launch": int(all_bytes / len(traces)) if traces else None,
                     "ms_per_launch": round(sweep_ms / len(traces), 4) if traces else None,
                     "bu_levels_gbs": round(bu_bytes / (bu_ms / 1e3) / 1e9, 1) if bu_ms else None,
                     "td_levels_gbs": round(td_bytes / (td_ms / 1e3) / 1e9, 1) if td_ms else None,
                     "bu_share_of_search_time": round(bu_ms / sweep_ms, 3) if sweep_ms else None},
        "e2e": e2e,
        "gpu_launches": int(launches_total),
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    line.update(extra)
    print(json.dumps(line), flush=True)


def e2e_dropin(lib, og, s, d, w, roots, rank, dev):
    """BFS through breadthFirstSearchGraphCSR on a host GraphCSR (built by
    graphCSRPreProcessingStep from a .wbin file): per call, the stats arrays
    are host malloc'd and parents/distances are copied device -> host."""
    import torch
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, f"rmat{SCALE}_{rank}.wbin")
    og.write_edge_file(path, s, d, w)
    a = og.default_arguments(fnameb=path, sort=0, weighted=1, pushpull=2)
    lib.initializeMersenneState(C.byref(a.mt19937var), 27491095)
    gh = lib.graphCSRPreProcessingStep(C.byref(a))
    V = gh.contents.num_vertices
    # warm-up
    for r in roots[:3]:
        a.source = r
        lib.freeBFSStats(lib.breadthFirstSearchGraphCSR(C.byref(a), gh))
    torch.cuda.synchronize()
    names = ("call", "stats_alloc", "device_search", "dual_sentinels", "search_and_sentinels",
             "result_copy")
    ph = (C.c_double * len(names))()
    acc = np.zeros(len(names))
    t0 = time.perf_counter()
    for r in roots:
        a.source = r
        lib.freeBFSStats(lib.breadthFirstSearchGraphCSR(C.byref(a), gh))
        lib.ogb_dropin_bfs_phases(ph, len(names))
        acc += np.frombuffer(ph, np.float64)
    t1 = time.perf_counter()
    phases_ms = {k: round(float(v) / len(roots) * 1e3, 4) for k, v in zip(names, acc)}
    # traversed edges of these roots (the same searches, run on the device copy)
    g = og.DeviceGraph(lib, handle=lib.ogb_graph_of(C.cast(gh, C.c_void_p)), owned=False)
    pt = torch.empty(V, dtype=torch.int32, device=dev)
    dt = torch.empty(V, dtype=torch.int32, device=dev)
    edges = sum(g.bfs(r, pt, dt, mode=2)["reached_out_edges"] for r in roots)
    lib.graphCSRFree(gh)
    os.remove(path)
    n = len(roots)
    return {"value": round(edges / (t1 - t0) / 1e9, 3), "unit": "GTEPS", "h2d_bytes_per_step": 0,
            "d2h_bytes_per_step": int(n * 8 * V), "calls_per_step": n,
            "ms_per_call": round((t1 - t0) / n * 1e3, 4), "phases_ms_per_call": phases_ms,
            "host_bytes_written_per_call": int(12 * V),
            "api": "breadthFirstSearchGraphCSR(pushpull=2) on a graphCSRPreProcessingStep GraphCSR"}


def stages(lib, og, g, ts, td, tw, V, E, dev, hbm_peak):
    import torch
    out = {}
    # ---- sort + CSR build (both directions, weighted) --------------------
    g2 = lib.device_graph()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        g2.build(ts, td, V, 0, weight=tw)
    torch.cuda.synchronize()
    times = []
    for _ in range(5):
        start.record()
        g2.build(ts, td, V, 0, weight=tw)
        stop.record()
        torch.cuda.synchronize()
        times.append(start.elapsed_time(stop))
    g2.close()
    build_ms = statistics.median(times)
    P = sort_passes(V)
    wgt = 1
    alg = 2 * ((16 + 4 * wgt) * E * P + 4 * E + 4 * E + 12 * V) + (16 + 8 * wgt) * E
    out["csr_build"] = {"ms": round(build_ms, 3), "medges_per_s": round(E / build_ms / 1e3, 1),
                        "algorithmic_gb": round(alg / 1e9, 3), "gbs": round(alg / build_ms / 1e6, 1),
                        "frac": round(alg / build_ms / 1e6 / hbm_peak, 4),
                        "note": "device sort+CSR both directions incl. one 8 KB host read per sort"}
    # ---- PageRank pull / push to 1e-6 -----------------------------------
    ranks = torch.empty(V, dtype=torch.float32, device=dev)
    for mode, name, per_edge in ((0, "pr_pull", 8), (1, "pr_push", 12)):
        # the first call on a graph also builds the per-graph lists (and, for
        # pull, the renumbered layout); measured as the extra time of call 1
        once = []
        for _ in range(2):
            start.record()
            g.pagerank(ranks, mode=mode, max_iterations=1, epsilon=0.0)
            stop.record()
            torch.cuda.synchronize()
            once.append(start.elapsed_time(stop))
        prepare_ms = max(once[0] - once[1], 0.0)
        for _ in range(3):
            g.pagerank(ranks, mode=mode, max_iterations=PR_MAX, epsilon=PR_TOL)
        torch.cuda.synchronize()
        info = g.pagerank(ranks, mode=mode, max_iterations=PR_MAX, epsilon=PR_TOL)
        errs, _ = g.pagerank_history()
        hit = next((i for i, e in enumerate(errs) if e < PR_TOL), None)
        # per-iteration time at a fixed count (no early exit)
        start.record()
        info20 = g.pagerank(ranks, mode=mode, max_iterations=20, epsilon=0.0)
        stop.record()
        torch.cuda.synchronize()
        it_ms = start.elapsed_time(stop) / 20
        alg = per_edge * E + 28 * V
        out[name] = {"ms_per_iteration": round(it_ms, 4), "gteps": round(E / it_ms / 1e6, 2),
                     "gbs": round(alg / it_ms / 1e6, 1), "frac": round(alg / it_ms / 1e6 / hbm_peak, 4),
                     "iterations_to_1e-6_l1": (hit + 1) if hit is not None else None,
                     "ms_to_1e-6_l1": round(it_ms * (hit + 1), 3) if hit is not None else None,
                     "reference_stop_rule_iterations": info["iterations"],
                     "device_ms_run": round(info["ms"], 3),
                     "prepare_ms_once_per_graph": round(prepare_ms, 3)}
    out["data_driven"] = data_driven(g, V, E, dev, hbm_peak)
    return out


def data_driven(g, V, E, dev, hbm_peak, eps=1e-4, max_iterations=PR_MAX):
    """Data-driven PageRank (pageRank.c:2405-2919) against the plain pull at
    OpenGraph's default epsilon, each run to the reference's stop rule, device
    time of the whole run (median of 3 after 2 warm runs); SPMV pull / push
    per iteration (SPMV.c:588-810, weighted graph) with their byte rooflines:
    pull 12 E + 16 V (in-edge id, weight, x gather; rows, y read + write),
    push 16 E + 12 V (out-edge id, weight, y atomic read + write; rows, x)."""
    import torch
    ranks = torch.empty(V, dtype=torch.float32, device=dev)
    res = {"epsilon": eps}
    for mode, name in ((0, "pull"), (6, "dd_pull"), (7, "dd_push"), (8, "dd_pullpush")):
        for _ in range(2):
            g.pagerank(ranks, mode=mode, max_iterations=max_iterations, epsilon=eps)
        runs = [g.pagerank(ranks, mode=mode, max_iterations=max_iterations, epsilon=eps) for _ in range(3)]
        ms = statistics.median(r["ms"] for r in runs)
        res[name] = {"ms": round(ms, 3), "iterations": runs[-1]["iterations"], "launches": runs[-1]["launches"]}
    res["dd_pull_vs_pull"] = round(res["pull"]["ms"] / res["dd_pull"]["ms"], 2)
    x = torch.empty(V, dtype=torch.float32, device=dev)
    y = torch.empty(V, dtype=torch.float32, device=dev)
    for mode, name, alg in ((0, "spmv_pull", 12 * E + 16 * V), (1, "spmv_push", 16 * E + 12 * V)):
        g.spmv(x, y, mode=mode, iterations=3)
        ms = statistics.median(g.spmv(x, y, mode=mode, iterations=20)["ms"] / 20 for _ in range(3))
        res[name] = {"ms_per_iteration": round(ms, 4), "gteps": round(E / ms / 1e6, 1),
                     "gbs": round(alg / ms / 1e6, 1), "frac": round(alg / ms / 1e6 / hbm_peak, 4)}
    return res


def batching(lib, og, g, roots, V, E, dev, sweep_ms, extra):
    """The batched paths on the same GPU: 64-root multi-source BFS against the
    64 single searches of the step, 32-seed personalized PageRank against 32
    single pull iterations, and 256 uneven small RMAT graphs (scales 10-17,
    edge factors 8-32) in one batch against the same graphs one by one."""
    import torch
    out = {}
    depth = torch.empty(V * 64, dtype=torch.int16, device=dev)
    for _ in range(2):
        g.msbfs(roots, depth)
    runs = [g.msbfs(roots, depth) for _ in range(3)]
    best = min(runs, key=lambda r: r["ms"])
    ms, init_ms = best["ms"], best["init_ms"]
    # like the single searches (whose output initialisation precedes their
    # timed region), `ms` is the search; init_ms (depth fill, word clears,
    # roots) is reported beside it and in the second ratio
    out["msbfs_64_roots"] = {"ms": round(ms, 3), "init_ms": round(init_ms, 3),
                             "sequential_64_searches_ms": round(sweep_ms, 3),
                             "speedup": round(sweep_ms / ms, 2),
                             "speedup_with_init": round(sweep_ms / (ms + init_ms), 2)}
    del depth
    rng = np.random.default_rng(5)
    seeds = [int(x) for x in rng.choice(V, size=32, replace=False)]
    ranks = torch.empty(V * 32, dtype=torch.float32, device=dev)
    g.ppr(seeds, ranks, max_iterations=3)
    info = g.ppr(seeds, ranks, max_iterations=20)
    it_ms = info["ms"] / 20
    single = extra.get("pr_pull", {}).get("ms_per_iteration")
    out["ppr_32_seeds"] = {"ms_per_iteration": round(it_ms, 3),
                           "seed_edge_updates_per_s": round(32 * E / it_ms / 1e6, 1),
                           "vs_32_single_iterations": round(32 * single / it_ms, 2) if single else None}
    del ranks
    lib_b = og.load(False)
    rng = np.random.default_rng(42)
    nv, srcs, dsts = [], [], []
    for i in range(256):
        sc, ef = int(rng.integers(10, 18)), int(rng.integers(8, 33))
        s_, d_, _ = og.generate_rmat(sc, ef, 5000 + i)
        nv.append(1 << sc)
        srcs.append(s_)
        dsts.append(d_)
    eoff = np.zeros(257, np.uint64)
    eoff[1:] = np.cumsum([len(x) for x in srcs])
    broots = [int(np.argmax(np.bincount(x, minlength=n))) for x, n in zip(srcs, nv)]
    b = og.GraphBatch(lib_b, nv, eoff, np.concatenate(srcs), np.concatenate(dsts))
    Vt = int(b.offsets[-1])
    par = torch.empty(Vt, dtype=torch.int32, device=dev)
    dis = torch.empty(Vt, dtype=torch.int32, device=dev)
    rk = torch.empty(Vt, dtype=torch.float32, device=dev)
    tune = b.autotune()
    b.bfs(broots, par, dis)
    bfs_ms = min(b.bfs(broots, par, dis)["ms"] for _ in range(3))
    b.pagerank(rk, max_iterations=100, epsilon=1e-4)
    pr_ms = min(b.pagerank(rk, max_iterations=100, epsilon=1e-4)[0]["ms"] for _ in range(2))
    gs = []
    for i in range(256):
        gi = lib_b.device_graph()
        gi.build(torch.from_numpy(srcs[i].view(np.int32)).to(dev), torch.from_numpy(dsts[i].view(np.int32)).to(dev),
                 nv[i], 0)
        gs.append(gi)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i, gi in enumerate(gs):
        gi.bfs(broots[i], par[:nv[i]], dis[:nv[i]], mode=2)
    torch.cuda.synchronize()
    seq_bfs = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    for i, gi in enumerate(gs):
        gi.pagerank(rk[:nv[i]], mode=0, max_iterations=100, epsilon=1e-4)
    torch.cuda.synchronize()
    seq_pr = (time.perf_counter() - t0) * 1e3
    for gi in gs:
        gi.close()
    b.close()
    best = tune["candidates"][tune["best"]]
    out["graphs_256"] = {"vertices": Vt, "edges": int(eoff[-1]), "bfs_ms": round(bfs_ms, 3),
                         "bfs_sequential_ms": round(seq_bfs, 2), "pagerank_ms": round(pr_ms, 2),
                         "pagerank_sequential_ms": round(seq_pr, 2),
                         "autotuned_bins": {"warp_thr": best[0], "cta_thr": best[1]},
                         "note": "sequential = the same graphs one by one through the single-graph API, wall clock"}
    return out


def learned_vs_plain(lib, og, g, roots, V, dev, flush, par, dis):
    """The learned parts against the plain ones on the bench graph: the same
    roots searched with the plain alpha/beta switch (mode 2) and the learned
    switch (mode 3), L2 flushed before each search, depths compared; and
    PageRank pull to the 1e-6 tolerance from the uniform start and from the
    warm-start network (its kernel timed in).  Held-out graphs (RMAT-24, a
    4096 x 4096 grid): python -m opengraph_b200.learned evaluate."""
    import torch

    from opengraph_b200 import learned
    sw = learned.load_weights(lib, learned.SWITCH)
    pw = learned.load_weights(lib, learned.PR_START)
    if sw is None or pw is None:
        return {"unavailable": "no trained weights in opengraph_b200/weights"}
    lib.check(lib.ogb_bfs_set_policy(sw.ctypes.data), "ogb_bfs_set_policy")
    out = {}
    try:
        res = {}
        same = True
        for mode, tag in ((2, "plain"), (3, "learned")):
            ms = edges = 0.0
            for i, r in enumerate(roots):
                flush.zero_()
                torch.cuda.synchronize()
                info = g.bfs(r, par, dis, mode=mode)
                ms += info["ms"]
                edges += info["reached_out_edges"]
                if i < 4:
                    dcopy = dis.cpu().numpy().copy()
                    if tag == "plain":
                        res.setdefault("depths", []).append(dcopy)
                    else:
                        same = same and np.array_equal(dcopy, res["depths"][i])
            res[tag] = {"gteps": round(edges / ms / 1e6, 2), "ms_per_search": round(ms / len(roots), 4)}
        out["bfs"] = {"plain": res["plain"], "learned": res["learned"], "depths_identical_first_4_roots": same}
        ranks = torch.empty(V, dtype=torch.float32, device=dev)
        init = torch.empty(V, dtype=torch.float32, device=dev)
        pr = {}
        for tag in ("plain", "learned"):
            for rep in range(2):   # the second run is reported
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record()
                if tag == "learned":
                    g.pagerank_warm_start(pw, init, hidden=learned.PR_START[2])
                info = g.pagerank(ranks, mode=0, max_iterations=200, epsilon=1e-6,
                                  init=init if tag == "learned" else None)
                ev1.record()
                torch.cuda.synchronize()
            pr[tag] = {"iterations": info["iterations"], "ms_to_1e-6": round(ev0.elapsed_time(ev1), 3),
                       "ranks": ranks.cpu().numpy().astype(np.float64)}
        l1 = float(np.abs(pr["plain"].pop("ranks") - pr["learned"].pop("ranks")).sum())
        pr["final_l1_between"] = l1
        out["pagerank_to_1e-6"] = pr
    finally:
        lib.ogb_bfs_set_policy(None)
    return out


def cpu_baseline(og, s, d, w, roots):
    """The reference's own OpenMP BFS (oracle/_ref, WEIGHTED build) on this
    host's cores, same .wbin graph, same roots."""
    from oracle.oracle import Reference
    if not Reference.available(True):
        return {"value": None, "unit": "GTEPS", "kind": "reference", "note": "oracle/_ref not built"}
    ref = Reference(True)
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, f"rmat{SCALE}.wbin")
    og.write_edge_file(path, s, d, w)
    cores = os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    t0 = time.perf_counter()
    rg = ref.build_graph(path, weighted_file=True)
    build_s = time.perf_counter() - t0
    ga_outdeg = og.as_numpy(rg.contents.vertices.contents.out_degree, rg.contents.num_vertices, np.uint32)
    edges, secs = 0, 0.0
    for r in roots:
        p, _, st = ref.bfs(rg, r, 2)
        edges += int(ga_outdeg[p >= 0].astype(np.uint64).sum())
        secs += st["time_total"]
    ref.graphCSRFree(rg)
    os.remove(path)
    return {"value": round(edges / secs / 1e9, 4), "unit": "GTEPS", "cores": cores, "kind": "reference",
            "sample": f"{len(roots)} of the {NROOTS} roots (DO-BFS, stats->time_total), same RMAT-{SCALE} graph",
            "csr_build_s": round(build_s, 3)}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    # This arm runs the reference alone: the input file is written by a
    # separate process (oracle/gen_rmat, the oracle's restatement of the
    # generator), so this process loads nothing but the reference's build.
    from oracle.oracle import HERE as ORACLE_DIR
    from oracle.oracle import Reference
    if not Reference.available(True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference CPU build) not present"}))
        return
    gen = os.path.join(ORACLE_DIR, "gen_rmat")
    if not os.path.exists(gen):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "gen_rmat"], check=True)
    V = 1 << SCALE
    ref = Reference(True)
    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, f"rmat{SCALE}.wbin")
    subprocess.run([gen, str(SCALE), str(EDGE_FACTOR), str(SEED), "1", path], check=True)
    cores = os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    rg = ref.build_graph(path, weighted_file=True)
    outdeg = np.ctypeslib.as_array(rg.contents.vertices.contents.out_degree, shape=(V,)).astype(np.uint32)
    rng = np.random.default_rng(1000)
    roots = [int(x) for x in rng.choice(np.nonzero(outdeg > 0)[0], size=NROOTS, replace=False)]
    per_step = args.cpu_roots

    def step(k):
        e, t = 0, 0.0
        for r in roots[(k * per_step) % NROOTS:][:per_step]:
            p, _, st = ref.bfs(rg, r, 2)
            e += int(outdeg[p >= 0].astype(np.uint64).sum())
            t += st["time_total"]
        return e, t

    for k in range(args.warmup):
        step(k)
    E_tot, T_tot = 0, 0.0
    for k in range(args.steps):
        e, t = step(k)
        E_tot += e
        T_tot += t
    ref.graphCSRFree(rg)
    os.remove(path)
    val = E_tot / T_tot / 1e9
    sample = f"{per_step} DO-BFS roots per step (of the {NROOTS}), RMAT-{SCALE}, reference stats->time_total"
    print(json.dumps({
        "metric": METRIC, "value": round(val, 4), "unit": "GTEPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(T_tot * 1e3 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded RMAT generator)",
        "config": dict(workload_config(ws), parallelism="openmp (reference CPU build, all host cores)"),
        "impl": "reference",
        "cpu_baseline": {"value": round(val, 4), "unit": "GTEPS", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(val, 4), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_scale(args):
    """The plain pipeline at the scaling sizes (unweighted uint32 ids): RMAT
    scale 26 (67 M vertices, 1.07 B edges) and Erdos-Renyi with 2^24
    vertices and 2^28 uniform edges.  Per graph: sort + CSR build of both
    directions, PageRank pull iterations and DO-BFS from 8 seeded roots (L2
    flushed before each search), each with its algorithmic GB/s and fraction
    of the measured HBM peak.  One JSON line."""
    import torch

    import opengraph_b200 as og
    dev = torch.device("cuda", 0)
    lib = og.load(False)
    lib.quiet(True)
    hbm_peak, peak_kind = peaks()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"case": "scale", "peak_gbs": hbm_peak, "peak_kind": peak_kind, "graphs": {}}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for name, gen, V in (("rmat26_ef16", lambda: og.generate_rmat(26, 16, 0)[:2], 1 << 26),
                         ("er24_m2^28", lambda: og.generate_uniform(1 << 24, 1 << 28, 0)[:2], 1 << 24)):
        t0 = time.perf_counter()
        s, d = gen()
        gen_s = time.perf_counter() - t0
        E = len(s)
        ts = torch.from_numpy(s.view(np.int32)).to(dev)
        td = torch.from_numpy(d.view(np.int32)).to(dev)
        del s, d
        g = lib.device_graph()
        g.build(ts, td, V, 0)
        torch.cuda.synchronize()
        times = []
        for _ in range(2):
            start.record()
            g.build(ts, td, V, 0)
            stop.record()
            torch.cuda.synchronize()
            times.append(start.elapsed_time(stop))
        build_ms = min(times)
        P = sort_passes(V)
        alg = 2 * (16 * E * P + 4 * E + 4 * E + 12 * V) + 16 * E
        res = {"V": V, "E": E, "host_generate_s": round(gen_s, 1),
               "csr_build": {"ms": round(build_ms, 2), "passes": P, "gbs": round(alg / build_ms / 1e6, 1),
                             "frac": round(alg / build_ms / 1e6 / hbm_peak, 4)}}
        del ts, td
        torch.cuda.empty_cache()
        ranks = torch.empty(V, dtype=torch.float32, device=dev)
        g.pagerank(ranks, mode=0, max_iterations=1, epsilon=0.0)   # builds the renumbered layout
        g.pagerank(ranks, mode=0, max_iterations=3, epsilon=0.0)
        start.record()
        g.pagerank(ranks, mode=0, max_iterations=10, epsilon=0.0)
        stop.record()
        torch.cuda.synchronize()
        it_ms = start.elapsed_time(stop) / 10
        alg = 8 * E + 28 * V
        res["pr_pull"] = {"ms_per_iteration": round(it_ms, 3), "gteps": round(E / it_ms / 1e6, 1),
                          "gbs": round(alg / it_ms / 1e6, 1), "frac": round(alg / it_ms / 1e6 / hbm_peak, 4)}
        del ranks
        outdeg = g.view(False).out_degree.cpu().numpy().view(np.uint32)
        roots = rank_roots(outdeg, 0, 8)
        par = torch.empty(V, dtype=torch.int32, device=dev)
        dis = torch.empty(V, dtype=torch.int32, device=dev)
        g.bfs(roots[0], par, dis, mode=2)
        ms = edges = nbytes = 0.0
        for r in roots:
            flush.zero_()
            torch.cuda.synchronize()
            info = g.bfs(r, par, dis, mode=2)
            ms += info["ms"]
            edges += info["reached_out_edges"]
            nbytes += bfs_bytes(g.bfs_trace(), V)[0]
        res["dobfs"] = {"roots": len(roots), "ms_per_search": round(ms / len(roots), 3),
                        "gteps": round(edges / ms / 1e6, 1), "gbs": round(nbytes / ms / 1e6, 1),
                        "frac": round(nbytes / ms / 1e6 / hbm_peak, 4)}
        del par, dis
        g.close()
        torch.cuda.empty_cache()
        out["graphs"][name] = res
        print(json.dumps({name: res}), file=sys.stderr, flush=True)
    print(json.dumps(out), flush=True)


def run_case(args):
    """One hot-path kernel family on its own, for profiler captures: `bfs`
    runs --n DO-BFS searches, `pr-pull` / `pr-push` one PageRank run of --n
    iterations, `pr-dd-pull` / `pr-dd-push` / `pr-dd-pullpush` one
    data-driven PageRank run of at most --n iterations at epsilon 1e-4,
    `spmv-pull` / `spmv-push` --n SPMV iterations, `build` --n sort + CSR
    builds, all on the seeded RMAT graph of --scale.  Prints one JSON line
    with the device times."""
    import torch
    import opengraph_b200 as og
    dev = torch.device("cuda", 0)
    lib = og.load(True)
    lib.quiet(True)
    s, d, w = og.generate_rmat(args.scale, EDGE_FACTOR, SEED, weighted=True)
    V, E = 1 << args.scale, len(s)
    ts = torch.from_numpy(s.view(np.int32)).to(dev)
    td = torch.from_numpy(d.view(np.int32)).to(dev)
    tw = torch.from_numpy(w).to(dev)
    g = lib.device_graph()
    out = {"case": args.case, "scale": args.scale, "V": V, "E": E, "n": args.n}
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.case == "build":
        times = []
        for _ in range(args.n):
            start.record()
            g.build(ts, td, V, 0, weight=tw)
            stop.record()
            torch.cuda.synchronize()
            times.append(round(start.elapsed_time(stop), 4))
        out["ms"] = times
    else:
        g.build(ts, td, V, 0, weight=tw)
        torch.cuda.synchronize()
        if args.case == "bfs":
            outdeg = g.view(False).out_degree.cpu().numpy().view(np.uint32)
            rng = np.random.default_rng(1000)
            roots = [int(x) for x in rng.choice(np.nonzero(outdeg > 0)[0], size=args.n, replace=False)]
            par = torch.empty(V, dtype=torch.int32, device=dev)
            dis = torch.empty(V, dtype=torch.int32, device=dev)
            res = []
            for r in roots:
                info = g.bfs(r, par, dis, mode=2)
                nbytes, _ = bfs_bytes(g.bfs_trace(), V)
                res.append({"root": r, "ms": round(info["ms"], 4), "algorithmic_bytes": int(nbytes),
                            "reached_out_edges": int(info["reached_out_edges"])})
            out["searches"] = res
        elif args.case.startswith("spmv"):
            x = torch.empty(V, dtype=torch.float32, device=dev)
            y = torch.empty(V, dtype=torch.float32, device=dev)
            info = g.spmv(x, y, mode=0 if args.case == "spmv-pull" else 1, iterations=args.n)
            out["ms_per_iteration"] = round(info["ms"] / max(args.n, 1), 4)
        elif args.case.startswith("pr-dd"):
            ranks = torch.empty(V, dtype=torch.float32, device=dev)
            mode = {"pr-dd-pull": 6, "pr-dd-push": 7, "pr-dd-pullpush": 8}[args.case]
            info = g.pagerank(ranks, mode=mode, max_iterations=args.n, epsilon=1e-4)
            out["ms"] = round(info["ms"], 3)
            out["iterations"] = info["iterations"]
        else:
            ranks = torch.empty(V, dtype=torch.float32, device=dev)
            mode = 0 if args.case == "pr-pull" else 1
            info = g.pagerank(ranks, mode=mode, max_iterations=args.n, epsilon=0.0)
            out["ms_per_iteration"] = round(info["ms"] / max(args.n, 1), 4)
    g.close()
    print(json.dumps(out), flush=True)


def run_bfs_partitioned(args):
    """--case bfs-part: the graph and the search partitioned over all ranks of
    the job (1-D vertex ranges, one process per GPU, NCCL; opengraph_b200.
    parallel).  Each rank starts from its shard of the seeded RMAT edge list
    of --scale and builds its part of the graph (split by owner, all-to-all,
    local sort + CSR: `build_ms`); then --n DO-BFS searches, each one search
    over all ranks.  Every phase is timed with CUDA events between barriers
    and the slowest rank's time is reported.  Also the split kernel alone on
    the rank's shard into 8 owners (`split`).  --fused: the searches' exchange
    fused into the steps (symmetric memory) instead of the all-reduces.
    Prints one JSON line (rank 0)."""
    import datetime

    import torch
    import torch.distributed as tdist
    import opengraph_b200 as og
    from opengraph_b200.parallel import (DeviceBfsRangeStep, DeviceEdgeSplit, SymmetricBfsBuffers, bfs_partitioned,
                                         partitioned_device_graph, shard_ranges)
    ws, rank, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    dist = tdist if ws > 1 else None
    if ws > 1 or args.fused:  # the fused exchange's symmetric memory needs a process group, even of one
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29531")
        tdist.init_process_group("nccl", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=120),
                                 device_id=dev)
    lib = og.load(True)
    lib.quiet(True)
    s, d, w = og.generate_rmat(args.scale, EDGE_FACTOR, SEED, weighted=True)
    V, E = 1 << args.scale, len(s)
    a, b = E * rank // ws, E * (rank + 1) // ws
    ts = torch.from_numpy(s[a:b].view(np.int32)).to(dev)
    td = torch.from_numpy(d[a:b].view(np.int32)).to(dev)
    tw = torch.from_numpy(w[a:b]).to(dev)
    del s, d, w
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        if ws > 1:
            tdist.barrier()
        torch.cuda.synchronize()
        start.record()
        out = fn()
        stop.record()
        torch.cuda.synchronize()
        t = torch.tensor([start.elapsed_time(stop)], dtype=torch.float64, device=dev)
        if ws > 1:
            tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        return out, float(t.item())

    ranges = shard_ranges(td, V, ws, dist)
    # the split alone, 8 owners (after one untimed call)
    b8 = [V * k // 8 for k in range(9)]
    splitter = DeviceEdgeSplit(lib)
    splitter.split(ts, td, tw, b8)
    sp, split_ms = timed(lambda: splitter.split(ts, td, tw, b8))
    split_bytes = 12 * int(ts.numel()) + 12 * sum(sp[3])
    del sp
    (g, Eg), build_ms = timed(lambda: partitioned_device_graph(lib, ts, td, tw, V, ranges, rank, ws, dist=dist))
    vf = g.view(False)
    lo, hi = ranges[rank]
    outdeg = np.zeros(V, np.int64)
    outdeg[lo:hi] = vf.out_degree.cpu().numpy().view(np.uint32)[lo:hi]
    if ws > 1:
        od = torch.from_numpy(outdeg).to(dev)
        tdist.all_reduce(od)
        outdeg = od.cpu().numpy()
    rng = np.random.default_rng(1000)
    roots = [int(x) for x in rng.choice(np.nonzero(outdeg > 0)[0], size=args.n + 1, replace=False)]
    step = DeviceBfsRangeStep(g)
    peers = SymmetricBfsBuffers(V, ranges, dev) if args.fused else None
    res = []
    for k, r in enumerate(roots):
        (par, dep, st), t = timed(lambda: bfs_partitioned(step, V, Eg, ranges, rank, ws, r, dev, dist=dist,
                                                          peers=peers))
        if k == 0:
            continue  # warm-up search
        reached_out = int(outdeg[par.cpu().numpy() >= 0].sum())
        res.append({"root": r, "ms": round(t, 4), "steps": len(st.directions), "bu_steps": st.bu_steps,
                    "gteps": round(reached_out / (t * 1e6), 2)})
    g.close()
    if rank == 0:
        print(json.dumps({"case": "bfs-part", "scale": args.scale, "V": V, "E": E, "n_gpus": ws,
                          "exchange": "fused (symmetric memory)" if args.fused else "all-reduce",
                          "ranges": [list(x) for x in ranges], "edges_per_rank": int(vf.num_edges),
                          "build_ms": round(build_ms, 3),
                          "split": {"owners": 8, "edges": int(ts.numel()), "ms": round(split_ms, 3),
                                    "algorithmic_bytes": split_bytes,
                                    "gbs": round(split_bytes / (split_ms * 1e6), 1)},
                          "searches": res,
                          "note": "each phase timed with CUDA events between barriers, max over ranks"}),
              flush=True)
    del peers
    if tdist.is_initialized():
        tdist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-roots", type=int, default=8)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-stages", action="store_true")
    ap.add_argument("--case", default="full", choices=["full", "bfs", "pr-pull", "pr-push", "pr-dd-pull", "pr-dd-push",
                                                     "pr-dd-pullpush", "spmv-pull", "spmv-push", "build", "scale", "bfs-part"],
                    help="full = the benchmark line; scale = the plain pipeline on RMAT-26 and ER-24; "
                         "bfs-part = one DO-BFS partitioned over all ranks; "
                         "the others run one kernel family for profiling")
    ap.add_argument("--scale", type=int, default=SCALE, help="RMAT scale of a --case run")
    ap.add_argument("--n", type=int, default=3, help="searches / iterations / builds of a --case run")
    ap.add_argument("--fused", action="store_true", help="bfs-part: the exchange fused into the steps")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.case == "scale":
        run_scale(args)
    elif args.case == "bfs-part":
        run_bfs_partitioned(args)
    elif args.case != "full":
        run_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
