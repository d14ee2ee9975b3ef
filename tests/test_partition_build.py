"""The graph build across ranks (opengraph_b200.parallel.exchange_edges) on
CPU, with the oracle's restatement of the stable split by owner: each rank
starts from its shard of the edge list and builds its graph from what it
receives.  For every vertex a rank owns, that graph's out-row and in-row
(destinations / sources and weights, in order) must equal the whole graph's
(graphCSR.c:107-248 on the concatenated shards), for sort types 0 and 1.
Then the partitioned DO-BFS and PageRank pull run on these partial graphs and
must give the oracle's single-process results (BFS.c:476-626,
pageRank.c:984-1044).  Ranks run as threads (ThreadDist) and as 2 gloo
processes.  No GPU."""
import os
import socket

import numpy as np
import pytest

from opengraph_b200.parallel import (bfs_partitioned, edge_balanced_ranges, exchange_edges,
                                     pagerank_pull_partitioned, shard_ranges)
from test_partition import OracleRangeStep
from test_partition_bfs import OracleBfsRangeStep, _roots, check_against_oracle, run_threads


class OracleEdgeSplit:
    """The oracle's split as the exchange's local step (CPU tensors)."""

    def __init__(self, oracle):
        self.o = oracle

    def split(self, src, dst, w, bounds):
        import torch
        s, d, ww, counts = self.o.partition_edges(src.numpy(), dst.numpy(), None if w is None else w.numpy(), bounds)
        return (torch.from_numpy(np.ascontiguousarray(s)), torch.from_numpy(np.ascontiguousarray(d)),
                None if ww is None else torch.from_numpy(np.ascontiguousarray(ww)), counts)


def shards(a, world):
    n = len(a)
    cut = [n * k // world for k in range(world + 1)]
    return [a[cut[k]: cut[k + 1]] for k in range(world)]


def rows(g, v, inverse):
    p = "i_" if inverse else "f_"
    a, n = int(g[p + "idx"][v]), int(g[p + "outdeg"][v])
    w = g.get(p + "w")
    return g[p + "dst"][a: a + n], (w[a: a + n] if w is not None else None)


def check_rows(whole, part, lo, hi):
    for inverse in (False, True):
        p = "i_" if inverse else "f_"
        assert np.array_equal(part[p + "outdeg"][lo:hi], whole[p + "outdeg"][lo:hi])
        for v in range(lo, hi):
            a, aw = rows(whole, v, inverse)
            b, bw = rows(part, v, inverse)
            assert np.array_equal(a, b), (v, inverse)
            if aw is not None:
                assert np.array_equal(aw.view(np.uint32), bw.view(np.uint32)), (v, inverse)


def _edges(oracle, weighted):
    s, d, w = oracle.generate_rmat(11, 8, 9)
    V = int(max(s.max(), d.max())) + 1
    rng = np.random.default_rng(3)
    # duplicates and self loops stay in, as the reference's build keeps them (no -k)
    extra = rng.integers(0, len(s), 500)
    s = np.concatenate([s, s[extra], np.arange(50, dtype=np.uint32)])
    d = np.concatenate([d, d[extra], np.arange(50, dtype=np.uint32)])
    w = rng.uniform(1, 64, len(s)).astype(np.float32) if weighted else None
    return s, d, w, V


def _build_rank(oracle, s, d, w, V, world, sort_type, r, dd):
    import torch
    ss, ds = shards(s, world), shards(d, world)
    ws = shards(w, world) if w is not None else [None] * world
    t = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    ranges = shard_ranges(t(ds[r]), V, world, dd)
    rs, rd, rw, E = exchange_edges(OracleEdgeSplit(oracle), t(ss[r]), t(ds[r]), t(ws[r]), ranges, r, world, dd)
    g = oracle.build(rs.numpy(), rd.numpy(), V, sort_type, w=None if rw is None else rw.numpy())
    return g, E, ranges


@pytest.mark.parametrize("world", [1, 2, 3, 5])
@pytest.mark.parametrize("sort_type,weighted", [(0, False), (1, False), (0, True)])
def test_partial_graphs_hold_whole_rows(oracle, world, sort_type, weighted):
    s, d, w, V = _edges(oracle, weighted)
    whole = oracle.build(s, d, V, sort_type, w=w)
    outs = run_threads(world, lambda r, dd: _build_rank(oracle, s, d, w, V, world, sort_type, r, dd))
    assert outs[0][2] == edge_balanced_ranges(whole["i_outdeg"], world)
    for r, (g, E, ranges) in enumerate(outs):
        assert E == len(s)
        lo, hi = ranges[r]
        check_rows(whole, g, lo, hi)
        # every edge is stored on its source's owner and, if another, its destination's
        assert g["num_edges"] <= 2 * len(s)


@pytest.mark.parametrize("world", [2, 3])
def test_searches_on_partial_graphs(oracle, world):
    s, d, _, V = _edges(oracle, False)
    whole = oracle.build(s, d, V, 0)
    outs = run_threads(world, lambda r, dd: _build_rank(oracle, s, d, None, V, world, 0, r, dd))
    graphs = [o[0] for o in outs]
    E, ranges = outs[0][1], outs[0][2]
    for root in _roots(whole, 2):
        res = run_threads(world, lambda r, dd: bfs_partitioned(OracleBfsRangeStep(oracle, graphs[r]), V, E, ranges,
                                                               r, world, root, "cpu", dist=dd))
        for par, dep, st in res:
            check_against_oracle(oracle, whole, root, 2, False, par.numpy(), dep.numpy(), st)
    oracle.set_gpu_order()
    want, info = oracle.pagerank(whole, 2, 60, 1e-7)
    res = run_threads(world, lambda r, dd: pagerank_pull_partitioned(OracleRangeStep(oracle, graphs[r]), V, ranges,
                                                                     r, world, 60, 1e-7, "cpu", dist=dd))
    for ranks, st in res:
        assert np.array_equal(ranks.numpy().view(np.uint32), want.view(np.uint32))
        assert st.iterations == info["iterations"]


def test_split_rejects_ids_past_the_ranges(oracle):
    with pytest.raises(ValueError):
        oracle.partition_edges(np.array([0, 9], np.uint32), np.array([1, 2], np.uint32), None, [0, 4, 8])


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        o = Oracle()
        s, d, w, V = _edges(o, True)
        g, E, ranges = _build_rank(o, s, d, w, V, world, 0, rank, dist)
        lo, hi = ranges[rank]
        whole = o.build(s, d, V, 0, w=w)
        check_rows(whole, g, lo, hi)
        root = _roots(whole, 1)[0]
        par, dep, st = bfs_partitioned(OracleBfsRangeStep(o, g), V, E, ranges, rank, world, root, "cpu", dist=dist)
        check_against_oracle(o, whole, root, 2, False, par.numpy(), dep.numpy(), st)
        np.save(os.path.join(out_dir, f"ok{rank}.npy"), np.array([1]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(600)
def test_two_ranks_gloo_build_and_search(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    assert all((tmp_path / f"ok{r}.npy").exists() for r in range(2))


def test_owned_rows_exact_for_random_shards_and_cuts(oracle):
    """Property: for random edge lists (duplicates and self loops included),
    random shard sizes and random owner cut points (empty ranges included),
    every rank's graph built from the exchanged edges holds the whole
    graph's out-rows and in-rows of its vertices, in order, for sort types 0
    and 1, with and without weights."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=60, deadline=None)
    @given(st.integers(1, 40), st.integers(0, 160), st.integers(1, 5), st.integers(0, 2**31 - 1),
           st.sampled_from([0, 1]), st.booleans())
    def check(V, E, world, seed, sort_type, weighted):
        import torch
        rng = np.random.default_rng(seed)
        s = rng.integers(0, V, E).astype(np.uint32)
        d = rng.integers(0, V, E).astype(np.uint32)
        w = rng.uniform(1, 9, E).astype(np.float32) if weighted else None
        cuts = np.sort(rng.integers(0, V + 1, world - 1))
        bounds = [0] + [int(c) for c in cuts] + [V]
        ranges = [(bounds[r], bounds[r + 1]) for r in range(world)]
        whole = oracle.build(s, d, V, sort_type, w=w)
        sc = np.sort(rng.integers(0, E + 1, world - 1))
        sb = [0] + [int(c) for c in sc] + [E]
        t = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731

        def body(r, dd):
            a, b = sb[r], sb[r + 1]
            rs, rd, rw, n = exchange_edges(OracleEdgeSplit(oracle), t(s[a:b]), t(d[a:b]),
                                           t(w[a:b]) if w is not None else None, ranges, r, world, dd)
            return oracle.build(rs.numpy(), rd.numpy(), V, sort_type, w=None if rw is None else rw.numpy()), n

        for r, (g, n) in enumerate(run_threads(world, body)):
            assert n == E
            check_rows(whole, g, *ranges[r])

    check()
