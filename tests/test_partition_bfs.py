"""The 1-D partitioned direction-optimizing BFS (opengraph_b200.parallel) on
CPU: the host loop (direction switch of BFS.c:546-587, exchange of the next
bytes, all-gather of the owned slices) with the oracle's restatement of one
range's step as the local step.  Depths, the step sequence and the stats
must equal the single-process oracle's (orc_bfs, BFS.c:476-626) exactly for
every partition; bottom-up parents too; top-down parents must be the
smallest in-neighbour one level up.  Partitions run as gloo ranks (2 processes) and as threads of
one process with an in-process exchange (ThreadDist, also used by the GPU
test).  No GPU."""
import os
import socket
import threading

import numpy as np
import pytest

from opengraph_b200.parallel import bfs_partitioned, edge_balanced_ranges


class ThreadDist:
    """torch.distributed's all_reduce / all_gather among the threads of one
    process (each thread sets ``local.rank``): test infrastructure that runs
    the ranks of a partition side by side.  A failing rank aborts the
    barrier, so the others end with an error instead of waiting."""

    class ReduceOp:
        SUM = "sum"
        MAX = "max"
        MIN = "min"

    def __init__(self, world: int):
        self.world = world
        self.bar = threading.Barrier(world, timeout=300)
        self.local = threading.local()
        self.slots = [None] * world

    def all_reduce(self, t, op="sum", group=None):
        import torch
        self.slots[self.local.rank] = t.clone()
        self.bar.wait()
        acc = self.slots[0].clone()
        for x in self.slots[1:]:
            acc = torch.maximum(acc, x) if op == "max" else torch.minimum(acc, x) if op == "min" else acc + x
        self.bar.wait()
        t.copy_(acc)

    def all_to_all_single(self, out, t, output_split_sizes=None, input_split_sizes=None, group=None):
        import torch
        r = self.local.rank
        ins = input_split_sizes or [t.numel() // self.world] * self.world
        starts = [sum(ins[:k]) for k in range(self.world)]
        self.slots[r] = [t[starts[k]: starts[k] + ins[k]].clone() for k in range(self.world)]
        self.bar.wait()
        got = [self.slots[k][r] for k in range(self.world)]
        self.bar.wait()
        out.copy_(torch.cat(got) if got else out)

    def all_gather(self, out, t, group=None):
        self.slots[self.local.rank] = t.clone()
        self.bar.wait()
        for i in range(self.world):
            out[i].copy_(self.slots[i])
        self.bar.wait()


def run_threads(world: int, body):
    """body(rank, dist) on `world` threads; returns their results by rank."""
    d = ThreadDist(world)
    out, errs = [None] * world, []

    def worker(r):
        d.local.rank = r
        try:
            out[r] = body(r, d)
        except BaseException as e:  # noqa: BLE001 -- re-raised below
            errs.append(e)
            d.bar.abort()

    ts = [threading.Thread(target=worker, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]
    return out


class OracleBfsRangeStep:
    """The oracle as one rank's step (CPU tensors): test infrastructure."""

    def __init__(self, oracle, g):
        self.o, self.g = oracle, g

    def init(self, lo, hi, root, parents, dist, frontier, visited, cand, counts):
        od = self.o.bfs_range_init(self.g, lo, hi, root, parents.numpy(), dist.numpy().view(np.uint32),
                                   frontier.numpy(), visited.numpy(), cand.numpy())
        counts.numpy()[:] = [1, od, 0, 0] if lo <= root < hi else [0, 0, 0, 0]

    def expand(self, lo, hi, direction, depth, frontier, visited, nxt, cand, parents, dist, counts):
        self.o.bfs_range_expand(self.g, lo, hi, direction, depth, frontier.numpy(), visited.numpy(), nxt.numpy(),
                                cand.numpy(), parents.numpy(), dist.numpy().view(np.uint32),
                                counts.numpy().view(np.uint64))

    def settle(self, lo, hi, direction, depth, cand, nxt, visited, parents, dist, counts):
        self.o.bfs_range_settle(self.g, lo, hi, direction, depth, cand.numpy(), nxt.numpy(), visited.numpy(),
                                parents.numpy(), dist.numpy().view(np.uint32), counts.numpy().view(np.uint64))


def check_against_oracle(oracle, g, root, mode, bitmap_nf, par, dep, res):
    """Partitioned result (numpy parents / depths, BfsPartitionResult) vs the
    single-process oracle."""
    ep, ed, st = oracle.bfs(g, root, mode, bitmap_nf)
    nsteps = st["td_steps"] + st["bu_steps"]
    assert res.iteration == st["iteration"] and res.processed_nodes == st["processed_nodes"]
    assert res.td_steps == st["td_steps"] and res.bu_steps == st["bu_steps"]
    assert list(res.directions[: len(st["dirs"])]) == [int(x) for x in st["dirs"]] and len(res.directions) == nsteps
    assert np.array_equal(dep.view(np.uint32), ed)
    reached = ep >= 0
    assert np.array_equal(par >= 0, reached)
    assert np.array_equal(par[~reached], ep[~reached])  # -out_degree / -1 of the reference's initialisation
    v = np.nonzero(reached)[0]
    v = v[v != root]
    assert par[root] == root
    if len(v):
        p = par[v].astype(np.int64)
        assert np.array_equal(dep[p].astype(np.int64), dep[v].astype(np.int64) - 1)
        # p -> v is an edge of the graph
        keys = np.sort((np.repeat(np.arange(len(g["f_outdeg"]), dtype=np.uint64), g["f_outdeg"].astype(np.int64))
                        << np.uint64(32)) | (g["f_dst"] & 0x3FFFFFFF).astype(np.uint64))
        want = (p.astype(np.uint64) << np.uint64(32)) | v.astype(np.uint64)
        pos = np.minimum(np.searchsorted(keys, want), len(keys) - 1)
        assert np.array_equal(keys[pos], want)
        bu = np.asarray(res.directions, np.int64)[dep[v].astype(np.int64) - 1] == 1
        assert np.array_equal(par[v[bu]], ep[v[bu]])  # bottom-up parents are the reference's
        # top-down parents: the smallest in-neighbour one level up
        src = np.repeat(np.arange(len(g["f_outdeg"]), dtype=np.int64), g["f_outdeg"].astype(np.int64))
        dst = (g["f_dst"] & 0x3FFFFFFF).astype(np.int64)
        dep64 = dep.astype(np.int64)
        up = reached[src] & reached[dst] & (dep64[src] == dep64[dst] - 1) & (dst != root)
        low = np.full(len(dep), np.iinfo(np.int64).max)
        np.minimum.at(low, dst[up], src[up])
        td = v[~bu]
        assert np.array_equal(par[td].astype(np.int64), low[td])


def _graph(oracle, kind, **kw):
    from conftest import graph_edges
    s, d, _, V = graph_edges(kind, **kw)
    return oracle.build(s, d, V, 0)


CASES = [("rmat", dict(scale=11, ef=16, seed=3)), ("grid", dict(side=40, p=0.02, seed=1)),
         ("star", dict(n=3000, seed=2)), ("chain", dict(n=400))]


def _roots(g, n=3, seed=5):
    od = g["f_outdeg"]
    rng = np.random.default_rng(seed)
    hub = int(np.argmax(od))
    nz = np.nonzero(od)[0]
    zero = np.nonzero(od == 0)[0]
    out = [hub, int(rng.choice(nz))]
    if len(zero):
        out.append(int(zero[0]))  # no out-edges: one empty top-down step
    return out[:n]


@pytest.mark.parametrize("kind,kw", CASES)
def test_single_rank_equals_oracle(oracle, kind, kw):
    g = _graph(oracle, kind, **kw)
    V, E = g["num_vertices"], g["num_edges"]
    step = OracleBfsRangeStep(oracle, g)
    for root in _roots(g):
        for mode, bitmap in ((2, False), (2, True), (0, False), (1, False)):
            par, dep, res = bfs_partitioned(step, V, E, [(0, V)], 0, 1, root, "cpu", mode=mode,
                                            bu_entry_nf_frontier=bitmap)
            check_against_oracle(oracle, g, root, mode, bitmap, par.numpy(), dep.numpy(), res)


@pytest.mark.parametrize("kind,kw", CASES)
@pytest.mark.parametrize("world", [2, 3, 5])
def test_thread_partitions_equal_oracle(oracle, kind, kw, world):
    g = _graph(oracle, kind, **kw)
    V, E = g["num_vertices"], g["num_edges"]
    ranges = edge_balanced_ranges(g["i_outdeg"], world)
    for root in _roots(g, 2):
        for mode in (2, 0, 1):
            outs = run_threads(world, lambda r, d: bfs_partitioned(OracleBfsRangeStep(oracle, g), V, E, ranges, r,
                                                                   world, root, "cpu", mode=mode, dist=d))
            for par, dep, res in outs:
                check_against_oracle(oracle, g, root, mode, False, par.numpy(), dep.numpy(), res)


def test_more_ranks_than_vertices(oracle):
    s = np.array([0, 1, 2, 2], np.uint32)
    d = np.array([1, 2, 0, 3], np.uint32)
    g = oracle.build(s, d, 5, 0)  # vertex 4 isolated
    ranges = edge_balanced_ranges(g["i_outdeg"], 8)
    assert any(lo == hi for lo, hi in ranges)
    for root in range(5):
        outs = run_threads(8, lambda r, dd: bfs_partitioned(OracleBfsRangeStep(oracle, g), 5, g["num_edges"], ranges,
                                                            r, 8, root, "cpu", dist=dd))
        for par, dep, res in outs:
            check_against_oracle(oracle, g, root, 2, False, par.numpy(), dep.numpy(), res)


def test_bad_arguments(oracle):
    g = _graph(oracle, "chain", n=50)
    step = OracleBfsRangeStep(oracle, g)
    with pytest.raises(ValueError):
        bfs_partitioned(step, 50, g["num_edges"], [(0, 50)], 0, 1, 50, "cpu")
    with pytest.raises(ValueError):
        bfs_partitioned(step, 50, g["num_edges"], [(0, 50)], 0, 1, 0, "cpu", mode=3)
    with pytest.raises(ValueError):
        bfs_partitioned(step, 50, g["num_edges"], [(0, 25), (25, 50)], 0, 2, 0, "cpu")


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        o = Oracle()
        g = _graph(o, "rmat", scale=12, ef=16, seed=4)
        V, E = g["num_vertices"], g["num_edges"]
        ranges = edge_balanced_ranges(g["i_outdeg"], world)
        for k, root in enumerate(_roots(g, 2)):
            par, dep, res = bfs_partitioned(OracleBfsRangeStep(o, g), V, E, ranges, rank, world, root, "cpu",
                                            dist=dist)
            np.save(os.path.join(out_dir, f"par{rank}_{k}.npy"), par.numpy())
            np.save(os.path.join(out_dir, f"dep{rank}_{k}.npy"), dep.numpy())
            np.save(os.path.join(out_dir, f"res{rank}_{k}.npy"),
                    np.array([res.iteration, res.processed_nodes, res.td_steps, res.bu_steps, *res.directions],
                             np.int64))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(600)
def test_two_ranks_gloo_equal_oracle(oracle, tmp_path):
    import torch.multiprocessing as mp

    from opengraph_b200.parallel import BfsPartitionResult
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    g = _graph(oracle, "rmat", scale=12, ef=16, seed=4)
    for k, root in enumerate(_roots(g, 2)):
        for r in range(world):
            par = np.load(str(tmp_path / f"par{r}_{k}.npy"))
            dep = np.load(str(tmp_path / f"dep{r}_{k}.npy"))
            x = np.load(str(tmp_path / f"res{r}_{k}.npy")).tolist()
            res = BfsPartitionResult(iteration=x[0], processed_nodes=x[1], td_steps=x[2], bu_steps=x[3],
                                     directions=x[4:], edges_examined=0, ranges=[])
            check_against_oracle(oracle, g, root, 2, False, par, dep, res)
