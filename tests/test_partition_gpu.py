"""GPU: the partitioned PageRank pull's local step (ogb_pagerank_range_*,
the CUDA kernel each rank runs) gives the single-GPU pull's ranks bit for
bit whatever the partition.  With one GPU here, the ranks of a 2- or 3-way
partition are run one after the other on the same device, each writing its
own slice of the shared next-contrib vector (what the all-gather of a real
run assembles); the 1-rank path goes through opengraph_b200.parallel.  The
multi-process exchange itself is tested over gloo in test_partition.py."""
import numpy as np
import pytest

from opengraph_b200.parallel import DeviceRangeStep, edge_balanced_ranges, pagerank_pull_partitioned
from test_build_gpu import dev, host

pytestmark = pytest.mark.gpu


def emulate_parts(torch, lib, dg, V, ranges, iters, eps):
    step = DeviceRangeStep(dg, "cuda")
    ranks = torch.empty(V, dtype=torch.float32, device="cuda")
    c = torch.empty(V, dtype=torch.float32, device="cuda")
    cn = torch.empty(V, dtype=torch.float32, device="cuda")
    step.init(ranks, c)
    it, executed = iters, 0
    for k in range(iters):
        err = act = 0
        for lo, hi in ranges:
            e, a = step.step(lo, hi, c, ranks, cn, eps)
            err += e
            act += a
        c, cn = cn, c
        executed = k + 1
        if act == 0:
            it = k
            break
    step.finish(ranks)
    return ranks, it, executed


@pytest.mark.parametrize("kind,kw", [("rmat", dict(scale=16, ef=16, seed=0)), ("star", dict(n=20_000, seed=4)),
                                     ("grid", dict(side=80, p=0.01, seed=2))])
def test_partitions_equal_single_gpu_pull(torch_cuda, lib, oracle, graphs, kind, kw):
    torch = torch_cuda
    s, d, _, V = graphs(kind, **kw)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    ref = torch.empty(V, dtype=torch.float32, device="cuda")
    for iters, eps in ((40, 1e-5), (100, 1e-7)):
        info = dg.pagerank(ref, mode=0, max_iterations=iters, epsilon=eps)
        want = host(ref, np.float32).view(np.uint32)
        for parts in (1, 2, 3):
            ranges = edge_balanced_ranges(g["i_outdeg"], parts)
            ranks, it, ex = emulate_parts(torch, lib, dg, V, ranges, iters, eps)
            assert np.array_equal(host(ranks, np.float32).view(np.uint32), want), (parts, iters)
            assert it == info["iterations"] and ex == info["executed"], (parts, it, info)
        ranks, res = pagerank_pull_partitioned(DeviceRangeStep(dg, "cuda"), V, [(0, V)], 0, 1, iters, eps, "cuda")
        assert np.array_equal(host(ranks, np.float32).view(np.uint32), want)
        assert res.iterations == info["iterations"]
    dg.close()


def test_range_step_rejects_bad_ranges(torch_cuda, lib, graphs):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=10, ef=8, seed=0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    step = DeviceRangeStep(dg, "cuda")
    x = torch.zeros(V, dtype=torch.float32, device="cuda")
    with pytest.raises(Exception):
        step.step(0, V + 1, x, x.clone(), x.clone(), 1e-4)
    with pytest.raises(Exception):
        step.step(5, 3, x, x.clone(), x.clone(), 1e-4)
    dg.close()
