"""Generate tests/golden/law_enron.npz: the reference's own equivalence-test
input and what the reference's CPU build computes on it.

The reference's equivalence test (00_graph_bench/src/tests/
test_open-graph-match.c:59-86) reads 01_test_graphs/LAW/LAW-enron/graph.bin
with dflag=1 (duplicates and self loops removed), sort=1, 100 iterations,
epsilon 1e-4, and draws its roots with MT19937 seeded 27491095 (one
generateRandInt for the trial count, then generateRandomRootGraphCSR per
trial).  This script runs the same calls on the reference's own OpenMP build
(oracle/_ref/libogref.so) and stores:

  * the input edge records (src, dst), so the GPU test needs no mounted
    reference tree;
  * SHA-256 digests of the twelve CSR arrays graphCSRPreProcessingStep
    returns (forward and inverse src/dst/out_degree/in_degree/edges_idx);
  * the first 8 roots of that draw, and per root and BFS pushpull 0/1/2 the
    distances digest, processed_nodes and iteration (pull parents digest too:
    the pull step's parent choice is deterministic, BFS.c:736-748);
  * PageRank pull and push ranks with their iteration count and error.

Run where the reference tree is mounted:  python tests/golden/make_law_enron.py
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import opengraph_b200 as og  # noqa: E402
from oracle.oracle import REFERENCE_ROOT, Reference  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "law_enron.npz")
LAW_ENRON = os.path.join(REFERENCE_ROOT, "01_test_graphs/LAW/LAW-enron/graph.bin")
CSR_KEYS = ("f_src", "f_dst", "f_outdeg", "f_indeg", "f_idx", "i_src", "i_dst", "i_outdeg", "i_indeg", "i_idx")
NROOTS = 8


def digest(a: np.ndarray) -> np.ndarray:
    """SHA-256 of the array's little-endian bytes, as 32 uint8."""
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<")).tobytes())
                         .digest(), np.uint8).copy()


def main():
    raw = np.fromfile(LAW_ENRON, dtype="<u4").reshape(-1, 2)
    ref = Reference(False)
    g = ref.build_graph(LAW_ENRON, sort=1, dflag=1)
    ga = og.graph_arrays(g)
    out = {"src": raw[:, 0].copy(), "dst": raw[:, 1].copy(),
           "shape": np.array([ga["num_vertices"], ga["num_edges"], ga["avg_degree"]], np.uint32)}
    for k in CSR_KEYS:
        out["csr_" + k] = digest(ga[k])
    mt = og.mt19937state()
    ref.initializeMersenneState(C.byref(mt), 27491095)
    ref.d.generateRandInt(C.byref(mt))   # the trial count draw (test_open-graph-match.c:110)
    ref.d.generateRandomRootGraphCSR.restype = C.c_uint32
    roots = [int(ref.d.generateRandomRootGraphCSR(C.byref(mt), g)) for _ in range(NROOTS)]
    out["roots"] = np.array(roots, np.uint32)
    for i, r in enumerate(roots):
        for mode in (0, 1, 2):
            p, dist, st = ref.bfs(g, r, mode)
            out[f"bfs_m{mode}_r{i}_dist"] = digest(dist)
            out[f"bfs_m{mode}_r{i}_stats"] = np.array([st["processed_nodes"], st["iteration"]], np.uint32)
            if mode == 0:
                out[f"bfs_m{mode}_r{i}_par"] = digest(p)
    for mode, tag in ((0, "pull"), (1, "push")):
        pr, st = ref.pagerank(g, mode, 100, 1e-4)
        out[f"pr_{tag}_ranks"] = pr
        out[f"pr_{tag}_stats"] = np.array([st["iterations"]], np.uint32)
        out[f"pr_{tag}_error"] = np.array([st["error_total"]], np.float64)
    ref.graphCSRFree(g)
    np.savez_compressed(OUT, **out)
    print(OUT, os.path.getsize(OUT))


if __name__ == "__main__":
    main()
