"""Generate tests/golden/dd_spmv_rmat10.npz from the reference's own CPU
build: data-driven PageRank (pushpull 6, 7, 8; pageRank.c:2405-2919, run
with one kernel thread -- threaded, the reference's push loses updates and is
not reproducible), SPMV pull (SPMV.c:616-713) and radixSortEdgesByPageRank
(reorder.c:165-221), on a seeded RMAT scale-10 edge list stored in the
fixture.

Run where the reference build exists (oracle/_ref):
    python tests/golden/make_golden_dd.py
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
from oracle.oracle import Reference, silenced_stdout  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dd_spmv_rmat10.npz")


def main():
    s, d, _ = og.generate_rmat(10, 16, 11)
    ref = Reference(False)
    path = os.path.join(tempfile.mkdtemp(), "g.bin")
    og.write_edge_file(path, s, d)
    rg = ref.build_graph(path)
    V = rg.contents.num_vertices
    out = {"src": s, "dst": d}
    for mode in (6, 7, 8):
        a = ref.arguments(pushpull=mode, iterations=50, epsilon=1e-5)
        a.ker_numThreads = 1
        with silenced_stdout():
            st = ref.pageRankGraphCSR(C.byref(a), rg)
        out[f"dd{mode}_ranks"] = og.as_numpy(st.contents.pageRanks, V, np.float32)
        out[f"dd{mode}_stats"] = np.array([st.contents.iterations], np.uint32)
        out[f"dd{mode}_error"] = np.array([st.contents.error_total], np.float64)
        ref.freePageRankStats(st)
    a = ref.arguments(pushpull=0, iterations=3)
    with silenced_stdout():
        st = ref.SPMVGraphCSR(C.byref(a), rg)
    out["spmv_x"] = og.as_numpy(st.contents.vector_input, V, np.float32)
    out["spmv_y"] = og.as_numpy(st.contents.vector_output, V, np.float32)
    ref.freeSPMVStats(st)
    pr = out["dd6_ranks"].copy()
    lab = np.random.default_rng(5).permutation(V).astype(np.uint32)
    out["sort_labels_in"] = lab.copy()
    ref.radixSortEdgesByPageRank(pr.ctypes.data_as(og.f32p), lab.ctypes.data_as(og.u32p), V)
    out["sort_labels_out"] = lab
    ref.graphCSRFree(rg)
    np.savez_compressed(OUT, **out)
    print(OUT, os.path.getsize(OUT))


if __name__ == "__main__":
    main()
