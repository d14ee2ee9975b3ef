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


def test_fused_peer_stores_equal_all_gather(torch_cuda, lib, oracle, graphs):
    """ogb_pagerank_range_step_peers: each part stores its contribs into
    every rank's next buffer (three local buffers stand in for three ranks'
    symmetric memory); after every iteration all copies hold the whole
    vector, and the ranks equal the single-GPU pull bit for bit."""
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=15, ef=16, seed=3)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    ref = torch.empty(V, dtype=torch.float32, device="cuda")
    info = dg.pagerank(ref, mode=0, max_iterations=40, epsilon=1e-7)
    ranges = edge_balanced_ranges(g["i_outdeg"], 3)
    step = DeviceRangeStep(dg, "cuda")
    ranks = torch.empty(V, dtype=torch.float32, device="cuda")
    bufs = [[torch.full((V,), float("nan"), device="cuda") for _ in range(3)] for _ in range(2)]
    c0 = torch.empty(V, dtype=torch.float32, device="cuda")
    step.init(ranks, c0)
    for b in bufs[0]:
        b.copy_(c0)
    peers = [torch.tensor([b.data_ptr() for b in bs], dtype=torch.int64, device="cuda") for bs in bufs]
    cur, it = 0, 40
    for k in range(40):
        act = 0
        for r, (lo, hi) in enumerate(ranges):
            # rank r reads its own copy and writes its own next copy plus everyone's
            _, a = step.step(lo, hi, bufs[cur][r], ranks, bufs[cur ^ 1][r], 1e-7, peers=peers[cur ^ 1])
            act += a
        nxt = [host(b, np.float32) for b in bufs[cur ^ 1]]
        assert all(np.array_equal(nxt[0].view(np.uint32), x.view(np.uint32)) for x in nxt[1:]), k
        assert not np.isnan(nxt[0]).any(), k
        cur ^= 1
        if act == 0:
            it = k
            break
    step.finish(ranks)
    assert np.array_equal(host(ranks, np.float32).view(np.uint32), host(ref, np.float32).view(np.uint32))
    assert it == info["iterations"]
    with pytest.raises(Exception):  # peers given without their addresses
        lib.check(lib.ogb_pagerank_range_step_peers(dg.handle, 0, V, bufs[0][0].data_ptr(), ranks.data_ptr(),
                                                    bufs[1][0].data_ptr(), None, 2, 1e-7, step.err.data_ptr(),
                                                    step.act.data_ptr(), None), "x")
    dg.close()


def _fused_worker(rank, out_path, port):
    import datetime
    import os

    import torch
    import torch.distributed as dist

    import opengraph_b200 as og
    from conftest import graph_edges
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        lib = og.load(False)
        lib.quiet(True)
        s, d, _, V = graph_edges("rmat", scale=14, ef=16, seed=1)
        dg = lib.device_graph()
        dg.build(dev(torch, s), dev(torch, d), V, 0)
        ranks, res = pagerank_pull_partitioned(DeviceRangeStep(dg, "cuda"), V, [(0, V)], 0, 1, 50, 1e-7, "cuda",
                                               dist=dist, fused=True)
        ref = torch.empty(V, dtype=torch.float32, device="cuda")
        info = dg.pagerank(ref, mode=0, max_iterations=50, epsilon=1e-7)
        np.save(out_path, np.array([int(np.array_equal(host(ranks, np.float32).view(np.uint32),
                                                        host(ref, np.float32).view(np.uint32))),
                                    res.iterations, info["iterations"]]))
        dg.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_fused_exchange_through_symmetric_memory(torch_cuda, tmp_path):
    """pagerank_pull_partitioned(fused=True): the next-contrib buffers in
    torch's symmetric memory, the range step storing into every rank's copy,
    a barrier instead of the all-gather; one rank of an NCCL group here."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "fused.npy")
    mp.spawn(_fused_worker, args=(out, port), nprocs=1, join=True)
    ok, it, want = np.load(out).tolist()
    assert ok == 1 and it == want
