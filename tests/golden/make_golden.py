"""Generate tests/golden/*.npz from the reference's own CPU build.

Inputs are small seeded synthetic graphs (stored in the fixture, so the
fixtures do not depend on the generator); outputs come from the reference
OpenMP code compiled by oracle/Makefile (oracle/_ref/libogref*.so), called
through its public C API:

  * sortRunAlgorithms for SORT_TYPE 0..3 (sortRun.c:26-63),
  * graphCSRPreProcessingStep with dflag 0/1 (graphCSR.c:164-248),
  * breadthFirstSearchGraphCSR pushpull 0/1/2 from three roots (BFS.c:238-268):
    distances, pull-mode parents, processed_nodes, iteration,
  * pageRankGraphCSR pull (pageRank.c:939-1062): ranks, iterations, error.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import opengraph_b200 as og  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def inputs():
    rng = np.random.default_rng(2024)
    cases = {}
    s, d, w = og.generate_rmat(8, 8, 17, weighted=True)
    cases["rmat8"] = (s, d, w)
    s, d, w = og.generate_grid(12, 0.1, 3, weighted=True)
    cases["grid12"] = (s, d, w)
    n = 600
    s = np.concatenate([np.zeros(n, np.uint32), rng.integers(0, 40, n).astype(np.uint32),
                        np.arange(40, 60, dtype=np.uint32)])
    d = np.concatenate([rng.integers(0, 40, n).astype(np.uint32), np.zeros(n, np.uint32),
                        np.arange(40, 60, dtype=np.uint32)])  # self loops
    w = rng.uniform(1, 256, len(s)).astype(np.float32)
    cases["star_dup"] = (s, d, w)
    s = np.arange(299, dtype=np.uint32)
    cases["chain300"] = (s, s + 1, np.ones(299, np.float32))
    return cases


def edge_arrays(el):
    a = og.edge_list_arrays(el)
    return a["src"], a["dst"], a.get("w")


def main():
    tmp = tempfile.mkdtemp()
    for weighted in (False, True):
        ref = Reference(weighted)
        for name, (s, d, w) in inputs().items():
            out = {"src": s, "dst": d, "w": w}
            path = os.path.join(tmp, name + (".wbin" if weighted else ".bin"))
            og.write_edge_file(path, s, d, w if weighted else None)
            for sort in range(4):
                el = ref.readEdgeListsbin(path.encode(), 0, 0, 1 if weighted else 0)
                from oracle.oracle import silenced_stdout
                with silenced_stdout():
                    el = ref.sortRunAlgorithms(el, sort)
                ss, sd, sw = edge_arrays(el)
                out[f"sort{sort}_src"], out[f"sort{sort}_dst"] = ss, sd
                if weighted:
                    out[f"sort{sort}_w"] = sw
                ref.freeEdgeList(el)
            for sort in (0, 1):
                for dflag in (0, 1):
                    if dflag and sort == 0:
                        continue
                    g = ref.build_graph(path, sort=sort, dflag=dflag, weighted_file=weighted)
                    ga = og.graph_arrays(g)
                    tag = f"csr_s{sort}_d{dflag}_"
                    for k, v in ga.items():
                        out[tag + k] = np.asarray(v)
                    if sort == 0 and dflag == 0:
                        V = ga["num_vertices"]
                        roots = [int(np.argmax(ga["f_outdeg"])), 0, V // 2]
                        out["bfs_roots"] = np.array(roots, np.uint32)
                        for mode in (0, 1, 2):
                            for i, r in enumerate(roots):
                                p, dist, st = ref.bfs(g, r, mode)
                                out[f"bfs_m{mode}_r{i}_dist"] = dist
                                out[f"bfs_m{mode}_r{i}_stats"] = np.array([st["processed_nodes"], st["iteration"]],
                                                                          np.uint32)
                                if mode == 0:
                                    out[f"bfs_m{mode}_r{i}_par"] = p
                        pr, pst = ref.pagerank(g, 0, 20, 1e-4)
                        out["pr_pull_ranks"] = pr
                        out["pr_pull_stats"] = np.array([pst["iterations"]], np.uint32)
                        out["pr_pull_error"] = np.array([pst["error_total"]], np.float64)
                    ref.graphCSRFree(g)
            out = {k: v for k, v in out.items() if v is not None}
            fn = os.path.join(OUT, f"{name}_{'w1' if weighted else 'w0'}.npz")
            np.savez_compressed(fn, **out)
            print(fn, os.path.getsize(fn))


if __name__ == "__main__":
    main()
