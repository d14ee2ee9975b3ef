"""GPU: the graph build across ranks.  The library's stable split by owner
(ogb_partition_edges) equals the oracle's restatement bit for bit; graphs
built by each rank from the exchanged edges (partitioned_device_graph) hold
the whole graph's out-rows and in-rows of the vertices they own, in order;
and the partitioned DO-BFS and PageRank pull on those partial graphs give
the oracle's / the single-GPU results.  With one GPU here, the ranks are
threads of one process exchanging through ThreadDist; they meet only on the
host between launches."""
import numpy as np
import pytest

from opengraph_b200.parallel import (DeviceBfsRangeStep, DeviceEdgeSplit, DeviceRangeStep, bfs_partitioned,
                                     owner_bounds, pagerank_pull_partitioned, partitioned_device_graph,
                                     shard_ranges)
from test_build_gpu import dev, host
from test_partition_bfs import _roots, check_against_oracle, run_threads
from test_partition_build import shards

pytestmark = pytest.mark.gpu


def _csr(dg, inverse):
    v = dg.view(inverse)
    deg = host(v.out_degree).astype(np.int64)
    dst = host(v.dst)
    w = host(v.weight, np.float32) if v.weight is not None else None
    return deg, dst, w


def _owned_block(deg, dst, w, lo, hi):
    a = int(deg[:lo].sum())
    n = int(deg[lo:hi].sum())
    return dst[a: a + n], (w[a: a + n] if w is not None else None)


def _check_rows(whole, part, lo, hi):
    for inverse in (False, True):
        wd, wdst, ww = _csr(whole, inverse)
        pd, pdst, pw = _csr(part, inverse)
        assert np.array_equal(wd[lo:hi], pd[lo:hi]), inverse
        a, aw = _owned_block(wd, wdst, ww, lo, hi)
        b, bw = _owned_block(pd, pdst, pw, lo, hi)
        assert np.array_equal(a, b), inverse
        if aw is not None:
            assert np.array_equal(aw.view(np.uint32), bw.view(np.uint32)), inverse


def _rank_graphs(torch, lib, s, d, w, V, world, sort_type=0):
    ss, ds = shards(s, world), shards(d, world)
    ws = shards(w, world) if w is not None else [None] * world

    def body(r, dd):
        src, dst = dev(torch, ss[r]), dev(torch, ds[r])
        wt = dev(torch, ws[r]) if w is not None else None
        ranges = shard_ranges(dst, V, world, dd)
        g, E = partitioned_device_graph(lib, src, dst, wt, V, ranges, r, world, sort_type=sort_type, dist=dd)
        torch.cuda.synchronize()
        return g, E, ranges
    return run_threads(world, body)


@pytest.mark.parametrize("parts", [1, 2, 3, 7])
def test_split_equals_oracle(torch_cuda, lib, oracle, graphs, parts):
    torch = torch_cuda
    s, d, w, V = graphs("rmat", scale=14, ef=16, seed=5, weighted=True)
    g = oracle.build(s, d, V, 0)
    from opengraph_b200.parallel import edge_balanced_ranges
    bounds = owner_bounds(edge_balanced_ranges(g["i_outdeg"], parts))
    for shard in (slice(0, len(s)), slice(1000, 1000 + 40_000)):
        got = DeviceEdgeSplit(lib).split(dev(torch, s[shard]), dev(torch, d[shard]), dev(torch, w[shard]), bounds)
        es, ed, ew, ec = oracle.partition_edges(s[shard], d[shard], w[shard], bounds)
        n = sum(ec)
        assert got[3] == ec
        assert np.array_equal(host(got[0])[:n], es) and np.array_equal(host(got[1])[:n], ed)
        assert np.array_equal(host(got[2], np.uint32)[:n], ew.view(np.uint32))
    # ids past the last range are an error, not a write
    with pytest.raises(Exception):
        DeviceEdgeSplit(lib).split(dev(torch, s), dev(torch, d), None, [0, 10, 20])
    # an empty shard
    e = torch.zeros(0, dtype=torch.int32, device="cuda")
    assert DeviceEdgeSplit(lib).split(e, e, None, bounds)[3] == [0] * parts


@pytest.mark.parametrize("kind,kw,world", [("rmat", dict(scale=14, ef=16, seed=3), 2),
                                           ("rmat", dict(scale=14, ef=16, seed=3), 3),
                                           ("star", dict(n=20_000, seed=4), 3),
                                           ("grid", dict(side=80, p=0.01, seed=2), 4)])
def test_partial_graphs_and_searches(torch_cuda, lib, oracle, graphs, kind, kw, world):
    torch = torch_cuda
    s, d, _, V = graphs(kind, **kw)
    whole_o = oracle.build(s, d, V, 0)
    whole = lib.device_graph()
    whole.build(dev(torch, s), dev(torch, d), V, 0)
    outs = _rank_graphs(torch, lib, s, d, None, V, world)
    gs = [o[0] for o in outs]
    E, ranges = outs[0][1], outs[0][2]
    try:
        assert E == len(s)
        for r, g in enumerate(gs):
            _check_rows(whole, g, *ranges[r])
        for root in _roots(whole_o, 2):
            res = run_threads(world, lambda r, dd: bfs_partitioned(DeviceBfsRangeStep(gs[r]), V, E, ranges, r, world,
                                                                   root, "cuda", dist=dd))
            for par, dep, st in res:
                check_against_oracle(oracle, whole_o, root, 2, False, host(par, np.int32), host(dep, np.int32), st)
        ref = torch.empty(V, dtype=torch.float32, device="cuda")
        info = whole.pagerank(ref, mode=0, max_iterations=60, epsilon=1e-7)
        res = run_threads(world, lambda r, dd: pagerank_pull_partitioned(DeviceRangeStep(gs[r], "cuda"), V, ranges, r,
                                                                         world, 60, 1e-7, "cuda", dist=dd))
        for ranks, st in res:
            assert np.array_equal(host(ranks, np.float32).view(np.uint32), host(ref, np.float32).view(np.uint32))
            assert st.iterations == info["iterations"]
    finally:
        whole.close()
        for g in gs:
            g.close()


def test_partial_graphs_weighted_sorted_by_pair(torch_cuda, lib, graphs):
    torch = torch_cuda
    s, d, w, V = graphs("rmat", scale=15, ef=16, seed=8, weighted=True)
    whole = lib.device_graph()
    whole.build(dev(torch, s), dev(torch, d), V, 1, weight=dev(torch, w))
    outs = _rank_graphs(torch, lib, s, d, w, V, 3, sort_type=1)
    try:
        for r, (g, E, ranges) in enumerate(outs):
            _check_rows(whole, g, *ranges[r])
    finally:
        whole.close()
        for g, _, _ in outs:
            g.close()
