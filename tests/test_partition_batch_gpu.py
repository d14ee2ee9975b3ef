"""GPU: batched work across ranks.  msbfs_replicas (roots split over the
ranks, 64 per ogb_msbfs launch on each rank's copy of the graph) gives every
root the oracle's BFS depths (BFS.c:476-626; unreached 0xFFFF); ppr_replicas
gives each seed the same vector as a one-seed ogb_ppr, bit for bit.  With one
GPU here the ranks are threads of one process, each with its own copy of the
graph, exchanging through ThreadDist."""
import numpy as np
import pytest

from opengraph_b200.parallel import msbfs_replicas, ppr_replicas
from test_build_gpu import dev, host
from test_partition_bfs import run_threads

pytestmark = pytest.mark.gpu


def _graphs(torch, lib, s, d, V, n):
    out = []
    for _ in range(n):
        g = lib.device_graph()
        g.build(dev(torch, s), dev(torch, d), V, 0)
        out.append(g)
    return out


@pytest.mark.parametrize("world", [1, 2, 3])
def test_msbfs_replicas_equal_oracle(torch_cuda, lib, oracle, graphs, world):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=14, ef=16, seed=6)
    g = oracle.build(s, d, V, 0)
    rng = np.random.default_rng(2)
    roots = [int(x) for x in rng.choice(np.nonzero(g["f_outdeg"])[0], 150, replace=False)]  # 3 launches on 1 rank
    gs = _graphs(torch, lib, s, d, V, world)
    try:
        outs = run_threads(world, lambda r, dd: msbfs_replicas(gs[r], roots, r, world, dist=dd))
        for got in outs:
            got = host(got, np.uint16).reshape(len(roots), V)
            for i, root in enumerate(roots):
                par, dist, _ = oracle.bfs(g, root, 2)
                want = np.where(par >= 0, dist, 0xFFFF).astype(np.uint16)
                assert np.array_equal(got[i], want), (world, i)
    finally:
        for x in gs:
            x.close()


@pytest.mark.parametrize("world", [1, 3])
def test_ppr_replicas_equal_one_seed_runs(torch_cuda, lib, graphs, world):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=13, ef=16, seed=9)
    gs = _graphs(torch, lib, s, d, V, max(world, 1))
    seeds = list(range(0, 3 * 35, 3))  # 35 seeds: two launches on 1 rank
    try:
        outs = run_threads(world, lambda r, dd: ppr_replicas(gs[r], seeds, r, world, max_iterations=15, dist=dd))
        one = torch.empty(V * 32, dtype=torch.float32, device="cuda")
        want = []
        for x in seeds:
            gs[0].ppr([x], one, max_iterations=15)
            want.append(host(one, np.float32).reshape(V, 32)[:, 0].copy())
        for got in outs:
            got = host(got, np.float32).reshape(len(seeds), V)
            for i in range(len(seeds)):
                assert np.array_equal(got[i].view(np.uint32), want[i].view(np.uint32)), (world, i)
    finally:
        for x in gs:
            x.close()
