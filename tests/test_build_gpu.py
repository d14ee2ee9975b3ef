"""GPU parity: stable radix sort and CSR build (both directions) against the
oracle, bit-exact (reference: radixsort.c, countsort.c, vertex.c:204-325,
graphCSR.c:164-248).  All calls go through the C ABI (ogb_sort_edges,
ogb_graph_build)."""
import ctypes as C

import numpy as np
import pytest

import opengraph_b200 as og

pytestmark = pytest.mark.gpu


def dev(torch, a):
    if a is None:
        return None
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t, dtype=np.uint32):
    return t.cpu().numpy().view(dtype)


CASES = [
    ("rmat", dict(scale=12, ef=16, seed=1)),
    ("rmat", dict(scale=16, ef=16, seed=0)),          # the reference's small config (1M edges)
    ("uniform", dict(n=50_000, m=300_001, seed=3)),   # ragged tile count
    ("grid", dict(side=64, p=0.05, seed=2)),
    ("star", dict(n=20_000, seed=4)),                 # one hub, duplicates, self loops
    ("chain", dict(n=5000)),
]


@pytest.mark.parametrize("kind,kw", CASES, ids=[f"{k}-{i}" for i, (k, _) in enumerate(CASES)])
@pytest.mark.parametrize("sort_type", [0, 1, 2, 3])
@pytest.mark.parametrize("weighted", [False, True])
def test_sort_matches_oracle(torch_cuda, lib, oracle, graphs, kind, kw, sort_type, weighted):
    torch = torch_cuda
    s, d, w, V = graphs(kind, weighted=weighted, **kw)
    E = len(s)
    mode = 1 if sort_type in (1, 3) else 0
    es, ed, ew = oracle.sort(s, d, w, mode)
    ts, td, tw = dev(torch, s), dev(torch, d), dev(torch, w)
    os_ = torch.empty_like(ts)
    od = torch.empty_like(td)
    ow = torch.empty_like(tw) if w is not None else None
    lib.check(lib.ogb_sort_edges(ts.data_ptr(), td.data_ptr(), tw.data_ptr() if tw is not None else None, E,
                                 sort_type, os_.data_ptr(), od.data_ptr(), ow.data_ptr() if ow is not None else None,
                                 og._stream(None)), "sort")
    torch.cuda.synchronize()
    assert np.array_equal(host(os_), es)
    assert np.array_equal(host(od), ed)
    if w is not None:
        assert np.array_equal(host(ow, np.float32).view(np.uint32), ew.view(np.uint32))
    # the input is read only
    assert np.array_equal(host(ts), s) and np.array_equal(host(td), d)


@pytest.mark.parametrize("kind,kw", CASES, ids=[f"{k}-{i}" for i, (k, _) in enumerate(CASES)])
@pytest.mark.parametrize("sort_type", [0, 1])
def test_csr_build_matches_oracle(torch_cuda, lib, oracle, graphs, kind, kw, sort_type):
    torch = torch_cuda
    for weighted in (False, True):
        s, d, w, V = graphs(kind, weighted=weighted, **kw)
        exp = oracle.build(s, d, V, sort_type, w)
        g = lib.device_graph()
        g.build(dev(torch, s), dev(torch, d), V, sort_type, weight=dev(torch, w))
        torch.cuda.synchronize()
        for tag, inv in (("f", False), ("i", True)):
            v = g.view(inv)
            assert v.num_vertices == V and v.num_edges == len(s)
            assert np.array_equal(host(v.src), exp[tag + "_src"]), tag + "_src"
            assert np.array_equal(host(v.dst), exp[tag + "_dst"]), tag + "_dst"
            assert np.array_equal(host(v.out_degree), exp[tag + "_outdeg"]), tag + "_outdeg"
            assert np.array_equal(host(v.in_degree), exp[tag + "_indeg"]), tag + "_indeg"
            assert np.array_equal(host(v.edges_idx), exp[tag + "_idx"]), tag + "_idx"
            if w is not None:
                assert np.array_equal(host(v.weight, np.float32).view(np.uint32), exp[tag + "_w"].view(np.uint32))
        g.close()


def test_sort_edge_sizes(torch_cuda, lib, oracle):
    """E = 0, 1, tile boundaries +-1, all-equal keys, max id 2^30-1."""
    torch = torch_cuda
    rng = np.random.default_rng(5)
    for E in [1, 2, 4095, 4096, 4097, 8191, 65537]:
        for hi in [1, 7, 1 << 16, (1 << 30) - 1]:
            s = rng.integers(0, hi, E, dtype=np.uint64).astype(np.uint32)
            d = rng.integers(0, 1 << 20, E, dtype=np.uint64).astype(np.uint32)
            for sort_type in (0, 1):
                es, ed, _ = oracle.sort(s, d, None, 1 if sort_type == 1 else 0)
                ts, td = dev(torch, s), dev(torch, d)
                os_, od = torch.empty_like(ts), torch.empty_like(td)
                lib.check(lib.ogb_sort_edges(ts.data_ptr(), td.data_ptr(), None, E, sort_type, os_.data_ptr(),
                                             od.data_ptr(), None, og._stream(None)), "sort")
                assert np.array_equal(host(os_), es) and np.array_equal(host(od), ed), (E, hi, sort_type)
    # E = 0 is a no-op
    lib.check(lib.ogb_sort_edges(None, None, None, 0, 0, None, None, None, None), "sort0")


def test_build_rejects_out_of_range_ids(torch_cuda, lib):
    torch = torch_cuda
    s = np.array([0, 1, 9], np.uint32)
    d = np.array([1, 2, 3], np.uint32)
    g = lib.device_graph()
    with pytest.raises(Exception):
        g.build(dev(torch, s), dev(torch, d), 5, 0)   # id 9 >= V = 5
    g.close()


def test_repeat_build_is_deterministic(torch_cuda, lib, graphs):
    torch = torch_cuda
    s, d, w, V = graphs("rmat", scale=14, ef=16, seed=9, weighted=True)
    outs = []
    for _ in range(2):
        g = lib.device_graph()
        g.build(dev(torch, s), dev(torch, d), V, 0, weight=dev(torch, w))
        v = g.view(True)
        outs.append((host(v.src).copy(), host(v.dst).copy(), host(v.edges_idx).copy()))
        g.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
