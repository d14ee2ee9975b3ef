"""The .csr binary graph file (graphCSR.c:380-558): writeToBinFileGraphCSR
must produce the reference's bytes, readFromBinFileGraphCSR must read back
the reference's file into the same GraphCSR (both struct layouts).  Host
code: runs without a GPU (the device copy is then made on first use); the
GPU test runs the algorithms on the copy built while reading."""
import os

import numpy as np
import pytest

from test_parity_gpu import check_parents_full


def _graph_file(og, tmp_path, weighted):
    s, d, w = og.generate_rmat(12, 16, 6, weighted=True)
    path = str(tmp_path / ("g.wbin" if weighted else "g.bin"))
    og.write_edge_file(path, s, d, w if weighted else None)
    return path


@pytest.mark.parametrize("weighted", [False, True])
def test_write_equals_reference_bytes(og, lib, libw, ref, refw, tmp_path, weighted):
    L, R = (libw, refw) if weighted else (lib, ref)
    path = _graph_file(og, tmp_path, weighted)
    rg = R.build_graph(path, sort=1, weighted_file=weighted)
    L.writeToBinFileGraphCSR(str(tmp_path / "ours").encode(), rg)
    R.writeToBinFileGraphCSR(str(tmp_path / "theirs").encode(), rg)
    a = open(str(tmp_path / "ours.csr"), "rb").read()
    b = open(str(tmp_path / "theirs.csr"), "rb").read()
    assert len(a) == len(b) and a == b
    R.graphCSRFree(rg)


@pytest.mark.parametrize("weighted", [False, True])
def test_read_equals_reference(og, lib, libw, ref, refw, tmp_path, weighted):
    from oracle.oracle import silenced_stdout
    L, R = (libw, refw) if weighted else (lib, ref)
    path = _graph_file(og, tmp_path, weighted)
    rg = R.build_graph(path, sort=0, weighted_file=weighted)
    R.writeToBinFileGraphCSR(str(tmp_path / "g").encode(), rg)
    R.graphCSRFree(rg)
    f = str(tmp_path / "g.csr").encode()
    ours = L.readFromBinFileGraphCSR(f)
    with silenced_stdout():
        theirs = R.readFromBinFileGraphCSR(f)
    oa, ta = og.graph_arrays(ours), og.graph_arrays(theirs)
    for k, v in ta.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(oa[k].view(np.uint32), v.view(np.uint32)), k
        else:
            assert oa[k] == v, k
    assert not ours.contents.sorted_edges_array.contents.label_array
    if weighted:
        assert ours.contents.max_weight == theirs.contents.max_weight
    L.graphCSRFree(ours)
    R.graphCSRFree(theirs)


@pytest.mark.gpu
def test_read_then_bfs_and_pagerank_on_device_copy(og, lib, ref, oracle, tmp_path):
    """A graph read from .csr runs BFS (NULL label arrays: identity) and
    PageRank through the drop-in API on the device copy made while reading."""
    import ctypes as C
    path = _graph_file(og, tmp_path, False)
    rg = ref.build_graph(path, sort=0)
    ref.writeToBinFileGraphCSR(str(tmp_path / "g").encode(), rg)
    ref.graphCSRFree(rg)
    g = lib.readFromBinFileGraphCSR(str(tmp_path / "g.csr").encode())
    ga = og.graph_arrays(g)
    V = ga["num_vertices"]
    root = int(np.argmax(ga["f_outdeg"]))
    a = og.default_arguments(source=root, pushpull=2)
    st = lib.breadthFirstSearchGraphCSR(C.byref(a), g)
    dist = og.as_numpy(st.contents.distances, V, np.uint32)
    par = og.as_numpy(st.contents.parents, V, np.int32)
    lib.freeBFSStats(st)
    _, edist, _ = oracle.bfs(ga, root, 2)
    assert np.array_equal(dist, edist)
    check_parents_full(ga, root, par, dist)
    a = og.default_arguments(pushpull=0, iterations=20, epsilon=1e-4)
    st = lib.pageRankGraphCSR(C.byref(a), g)
    pr = og.as_numpy(st.contents.pageRanks, V, np.float32).astype(np.float64)
    it = st.contents.iterations
    lib.freePageRankStats(st)
    er, ei = oracle.pagerank(ga, 0, 20, 1e-4)
    assert it == ei["iterations"] and float(np.abs(pr - er).sum()) <= 1e-6
    lib.graphCSRFree(g)
