"""The 1-D partitioned PageRank pull (opengraph_b200.parallel) on CPU: the
partition and the exchange (all-gather of contrib slices, all-reduce of
error / active, the stop rule) over gloo with 2 ranks, each running the
oracle's restatement of one range's iteration (pageRank.c:984-1044 restricted
to the range, rows in the GPU kernels' summation order).  The ranks must equal
the single-process oracle's bit for bit, iteration count included.  No GPU."""
import os
import socket

import numpy as np
import pytest

from opengraph_b200.parallel import edge_balanced_ranges, pagerank_pull_partitioned


class OracleRangeStep:
    """The oracle as the local step (CPU tensors): test infrastructure."""

    def __init__(self, oracle, g):
        self.o, self.g = oracle, g

    def init(self, ranks, contrib):
        od = self.g["f_outdeg"]
        base = np.float32(1.0) - np.float32(0.85)
        ranks.numpy()[:] = base
        c = contrib.numpy()
        c[:] = 0.0
        nz = od > 0
        c[nz] = base / od[nz].astype(np.float32)

    def step(self, lo, hi, contrib, ranks, contrib_next, epsilon):
        return self.o.pull_range_step(self.g, lo, hi, contrib.numpy(), ranks.numpy(), contrib_next.numpy(),
                                      epsilon)

    def finish(self, ranks):
        r = ranks.numpy()
        r[:] = r / np.float32(self.g["num_vertices"])


def _graph(oracle):
    s, d, _ = oracle.generate_rmat(12, 16, 4)
    V = int(max(s.max(), d.max())) + 1
    return oracle.build(s, d, V, 0)


def test_edge_balanced_ranges():
    deg = np.random.default_rng(0).integers(0, 50, 10_000)
    deg[17] = 100_000  # one hub
    for parts in (1, 2, 3, 8):
        rs = edge_balanced_ranges(deg, parts)
        assert rs[0][0] == 0 and rs[-1][1] == len(deg)
        assert all(rs[k][1] == rs[k + 1][0] for k in range(parts - 1))
        work = [int((deg[l:h] + 1).sum()) for l, h in rs]
        # every range within one vertex's work of the even share, except where one row alone exceeds it
        share = (deg + 1).sum() / parts
        assert max(work) <= share + deg.max() + 1
    assert edge_balanced_ranges(np.zeros(0, np.int64), 2) == [(0, 0), (0, 0)]


def test_single_rank_equals_oracle(oracle):
    import torch
    g = _graph(oracle)
    V = g["num_vertices"]
    oracle.set_gpu_order()
    for iters, eps in ((25, 1e-5), (100, 1e-7)):
        ranks, res = pagerank_pull_partitioned(OracleRangeStep(oracle, g), V, [(0, V)], 0, 1, iters, eps, "cpu")
        er, ei = oracle.pagerank(g, 2, iters, eps)
        assert np.array_equal(ranks.numpy().view(np.uint32), er.view(np.uint32))
        assert res.iterations == ei["iterations"] and res.executed == ei["executed"]


def _worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        o = Oracle()
        o.set_gpu_order()
        g = _graph(o)
        V = g["num_vertices"]
        ranges = edge_balanced_ranges(g["i_outdeg"], world)
        ranks, res = pagerank_pull_partitioned(OracleRangeStep(o, g), V, ranges, rank, world, 100, 1e-7, "cpu",
                                               dist=dist)
        np.save(os.path.join(out_dir, f"ranks{rank}.npy"), ranks.numpy())
        np.save(os.path.join(out_dir, f"res{rank}.npy"),
                np.array([res.iterations, res.executed, res.active], np.int64))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(600)
def test_two_ranks_gloo_equal_single_rank(oracle, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    oracle.set_gpu_order()
    g = _graph(oracle)
    er, ei = oracle.pagerank(g, 2, 100, 1e-7)
    for r in range(world):
        got = np.load(str(tmp_path / f"ranks{r}.npy"))
        res = np.load(str(tmp_path / f"res{r}.npy"))
        assert np.array_equal(got.view(np.uint32), er.view(np.uint32)), r
        assert int(res[0]) == ei["iterations"] and int(res[1]) == ei["executed"], r


def test_random_graphs_and_cuts_bit_exact(oracle):
    """Property: random small graphs (duplicates, self loops, vertices
    without in- or out-edges), random owner cut points (empty ranges
    included), 1-4 thread-ranks: the partitioned pull equals the
    single-process oracle bit for bit, iteration count included."""
    from hypothesis import given, settings, strategies as st

    from test_partition_bfs import run_threads
    oracle.set_gpu_order()

    @settings(max_examples=30, deadline=None)
    @given(st.integers(2, 60), st.integers(1, 300), st.integers(1, 4), st.integers(0, 2**31 - 1))
    def check(V, E, world, seed):
        rng = np.random.default_rng(seed)
        s = rng.integers(0, V, E).astype(np.uint32)
        d = rng.integers(0, V, E).astype(np.uint32)
        g = oracle.build(s, d, V, 0)
        cuts = np.sort(rng.integers(0, V + 1, world - 1))
        bounds = [0] + [int(c) for c in cuts] + [V]
        ranges = [(bounds[r], bounds[r + 1]) for r in range(world)]
        want, info = oracle.pagerank(g, 2, 50, 1e-7)
        outs = run_threads(world, lambda r, dd: pagerank_pull_partitioned(OracleRangeStep(oracle, g), V, ranges, r,
                                                                          world, 50, 1e-7, "cpu",
                                                                          dist=dd if world > 1 else None))
        for ranks, res in outs:
            assert np.array_equal(ranks.numpy().view(np.uint32), want.view(np.uint32))
            assert res.iterations == info["iterations"] and res.executed == info["executed"]

    check()
