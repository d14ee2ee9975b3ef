"""CPU tests of the C-ABI boundary: the libraries load, export every symbol
that include/*.h declares, keep the reference struct layouts, and their host
functions (edge-list I/O, MT19937, root picker) match the reference's own
build.  No CUDA call is made here."""
import ctypes as C
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for f in os.listdir(INCLUDE):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "sizeof", "return"):
                names.add(name)
    return names


@pytest.mark.parametrize("weighted", [False, True])
def test_library_exports_every_declared_symbol(og, weighted):
    lib = og.load(weighted)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib.dll, n)]
    assert not missing, missing
    assert lib.ogb_weighted_layout() == int(weighted)


def test_declared_functions_are_many():
    names = declared_functions()
    for n in ("graphCSRPreProcessingStep", "sortRunAlgorithms", "breadthFirstSearchGraphCSR", "pageRankGraphCSR",
              "topDownStepGraphCSR", "bottomUpStepGraphCSR", "ogb_bfs", "ogb_graph_build"):
        assert n in names


def _probe(weighted):
    p = os.path.join(ROOT, "oracle", "_ref", f"layout_w{1 if weighted else 0}.txt")
    if not os.path.exists(p):
        pytest.skip("layout probe of the reference headers not built")
    out = {}
    for line in open(p):
        k, v = line.split()
        out[k] = int(v)
    return out


@pytest.mark.parametrize("weighted", [False, True])
def test_struct_layouts_match_reference_headers(og, weighted):
    probe = _probe(weighted)
    classes = {"Arguments": og.Arguments, "EdgeList": og.EdgeListW if weighted else og.EdgeList,
               "Vertex": og.Vertex, "GraphCSR": og.GraphCSRW if weighted else og.GraphCSR,
               "BFSStats": og.BFSStats, "PageRankStats": og.PageRankStats, "Bitmap": og.Bitmap,
               "ArrayQueue": og.ArrayQueue}
    for key, val in probe.items():
        if key == "mt19937state":
            assert C.sizeof(og.mt19937state) == val
            continue
        if "." in key:
            s, f = key.split(".")
            assert getattr(classes[s], f).offset == val, key
        else:
            assert C.sizeof(classes[key]) == val, key


def test_header_layout_compiles_identically(tmp_path):
    """include/ogb200.h compiled by a C compiler gives the probe's layout."""
    probe0 = _probe(False)
    for w in (0, 1):
        src = tmp_path / f"p{w}.c"
        src.write_text(
            f'#define OGB200_WEIGHTED {w}\n#include "ogb200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
            'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(struct Arguments), sizeof(struct EdgeList),'
            ' sizeof(struct GraphCSR), offsetof(struct EdgeList, edges_array_src), sizeof(struct BFSStats));}\n')
        exe = tmp_path / f"p{w}"
        subprocess.run(["gcc", "-I", INCLUDE, str(src), "-o", str(exe)], check=True)
        vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
        probe = probe0 if w == 0 else _probe(True)
        assert vals == [probe["Arguments"], probe["EdgeList"], probe["GraphCSR"], probe["EdgeList.edges_array_src"],
                        probe["BFSStats"]]


def test_mt19937_matches_reference(og, lib, ref, oracle):
    a, b = og.mt19937state(), og.mt19937state()
    lib.initializeMersenneState(C.byref(a), 27491095)
    ref.initializeMersenneState(C.byref(b), 27491095)
    for _ in range(3000):
        assert lib.generateRandInt(C.byref(a)) == ref.generateRandInt(C.byref(b))
    for _ in range(100):
        x, y = lib.generateRandFloat(C.byref(a)), ref.generateRandFloat(C.byref(b))
        assert np.float32(x).view(np.uint32) == np.float32(y).view(np.uint32)


@pytest.fixture(scope="module")
def edge_file(tmp_path_factory, og, graphs):
    d = tmp_path_factory.mktemp("abi")
    s, dd, w, V = graphs("rmat", scale=10, ef=16, seed=3, weighted=True)
    p, pw = str(d / "g.bin"), str(d / "g.wbin")
    og.write_edge_file(p, s, dd)
    og.write_edge_file(pw, s, dd, w)
    return p, pw


@pytest.mark.parametrize("weighted_layout", [False, True])
@pytest.mark.parametrize("inverse,symmetric,weighted_file", [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)])
def test_read_edge_lists_match_reference(og, ref, refw, edge_file, weighted_layout, inverse, symmetric,
                                         weighted_file):
    lib = og.load(weighted_layout)
    R = refw if weighted_layout else ref
    path = edge_file[1] if weighted_file else edge_file[0]
    o = lib.readEdgeListsbin(path.encode(), inverse, symmetric, weighted_file)
    t = R.readEdgeListsbin(path.encode(), inverse, symmetric, weighted_file)
    oa, ta = og.edge_list_arrays(o), og.edge_list_arrays(t)
    for k in ta:
        if isinstance(ta[k], np.ndarray):
            assert np.array_equal(oa[k].view(np.uint32), ta[k].view(np.uint32)), k
        else:
            assert oa[k] == ta[k], k
    V = o.contents.num_vertices
    assert np.array_equal(og.as_numpy(o.contents.label_array, V, np.uint32), np.arange(V))
    for inv in (0, 1):
        om = lib.readEdgeListsMem(o, inv, 0, 0)
        tm = R.readEdgeListsMem(t, inv, 0, 0)
        a, b = og.edge_list_arrays(om), og.edge_list_arrays(tm)
        for k in b:
            if isinstance(b[k], np.ndarray):
                assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k
        lib.freeEdgeList(om)
        R.freeEdgeList(tm)
    lib.freeEdgeList(o)
    R.freeEdgeList(t)


def test_new_structs_are_zeroed(og, lib):
    e = lib.newEdgeList(1000)
    assert e.contents.num_edges == 1000 and e.contents.num_vertices == 0
    assert not og.as_numpy(e.contents.edges_array_src, 1000, np.uint32).any()
    assert not e.contents.label_array
    lib.freeEdgeList(e)
    g = lib.graphCSRNew(100, 1000, 1)
    assert g.contents.avg_degree == 10 and bool(g.contents.inverse_vertices)
    assert not og.as_numpy(g.contents.vertices.contents.edges_idx, 100, np.uint32).any()
    lib.graphCSRFree(g)


def test_random_root_matches_reference(og, lib, ref, edge_file):
    rg = ref.build_graph(edge_file[0])
    a, b = og.mt19937state(), og.mt19937state()
    lib.initializeMersenneState(C.byref(a), 27491095)
    ref.initializeMersenneState(C.byref(b), 27491095)
    for _ in range(50):
        assert lib.generateRandomRootGraphCSR(C.byref(a), rg) == ref.d.generateRandomRootGraphCSR(C.byref(b), rg)
    ref.graphCSRFree(rg)


def test_missing_file_exits_like_reference(tmp_path):
    """readEdgeListsbin on a missing file: err(1) -- message and exit status 1."""
    code = ("import ctypes, sys; sys.path.insert(0, %r); import opengraph_b200 as og; "
            "lib = og.load(False); lib.readEdgeListsbin(b'/nonexistent/x.bin', 0, 0, 0)" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert r.returncode == 1
    assert "open: /nonexistent/x.bin" in r.stderr


def test_generators_are_deterministic(og):
    a = og.generate_rmat(12, 8, 5, weighted=True)
    b = og.generate_rmat(12, 8, 5, weighted=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    s, d, w = a
    assert s.max() < 4096 and d.max() < 4096 and w.min() >= 1.0 and w.max() < 256.0
    s, d, _ = og.generate_grid(8, 1.0, 0)
    assert len(s) == 4 * 8 * 7 + 2 * 49
