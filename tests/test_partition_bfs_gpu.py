"""GPU: the partitioned DO-BFS step kernels (ogb_bfs_range_*) under the host
loop of opengraph_b200.parallel.  Depths, the step sequence and the stats
equal the oracle's single search (orc_bfs, BFS.c:476-626) for every
partition, bottom-up parents too, top-down parents are the smallest
in-neighbour one level up; and the depths equal the single-GPU search's.  With one GPU here, the
ranks of a partition run as threads of one process, each with its own copy
of the graph and its own frontier / visited bytes, exchanging through
ThreadDist (the all-reduce and all-gather of a real run, done by torch ops on
the device).  No kernel waits on another rank's: the ranks meet only on the
host between launches."""
import numpy as np
import pytest

from opengraph_b200.parallel import DeviceBfsRangeStep, bfs_partitioned, edge_balanced_ranges
from test_build_gpu import dev, host
from test_partition_bfs import _roots, check_against_oracle, run_threads

pytestmark = pytest.mark.gpu

CASES = [("rmat", dict(scale=14, ef=16, seed=3)), ("grid", dict(side=80, p=0.01, seed=2)),
         ("star", dict(n=20_000, seed=4)), ("chain", dict(n=600)), ("uniform", dict(n=30_000, m=200_000, seed=1))]


def _device_graphs(torch, lib, s, d, V, n):
    gs = []
    for _ in range(n):
        dg = lib.device_graph()
        dg.build(dev(torch, s), dev(torch, d), V, 0)
        gs.append(dg)
    return gs


@pytest.mark.parametrize("kind,kw", CASES)
def test_partitions_equal_oracle(torch_cuda, lib, oracle, graphs, kind, kw):
    torch = torch_cuda
    s, d, _, V = graphs(kind, **kw)
    g = oracle.build(s, d, V, 0)
    E = g["num_edges"]
    gs = _device_graphs(torch, lib, s, d, V, 3)
    try:
        for root in _roots(g):
            for mode in (2, 0, 1):
                par, dep, res = bfs_partitioned(DeviceBfsRangeStep(gs[0]), V, E, [(0, V)], 0, 1, root, "cuda",
                                                mode=mode)
                check_against_oracle(oracle, g, root, mode, False, host(par, np.int32), host(dep, np.int32), res)
            for world in (2, 3):
                ranges = edge_balanced_ranges(g["i_outdeg"], world)
                outs = run_threads(world, lambda r, dd: bfs_partitioned(DeviceBfsRangeStep(gs[r]), V, E, ranges, r,
                                                                        world, root, "cuda", dist=dd))
                for par, dep, res in outs:
                    check_against_oracle(oracle, g, root, 2, False, host(par, np.int32), host(dep, np.int32), res)
            # the single-GPU search: the same depths
            p1 = torch.empty(V, dtype=torch.int32, device="cuda")
            d1 = torch.empty(V, dtype=torch.int32, device="cuda")
            gs[0].bfs(root, p1, d1, mode=2)
            assert np.array_equal(host(d1, np.int32), host(dep, np.int32))
    finally:
        for dg in gs:
            dg.close()


def test_partitions_rmat18_four_ranks(torch_cuda, lib, oracle, graphs):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=18, ef=16, seed=7)
    g = oracle.build(s, d, V, 0)
    E = g["num_edges"]
    gs = _device_graphs(torch, lib, s, d, V, 4)
    try:
        ranges = edge_balanced_ranges(g["i_outdeg"], 4)
        for root in _roots(g, 2):
            outs = run_threads(4, lambda r, dd: bfs_partitioned(DeviceBfsRangeStep(gs[r]), V, E, ranges, r, 4, root,
                                                                "cuda", dist=dd))
            for par, dep, res in outs:
                check_against_oracle(oracle, g, root, 2, False, host(par, np.int32), host(dep, np.int32), res)
    finally:
        for dg in gs:
            dg.close()


def test_range_calls_reject_bad_arguments(torch_cuda, lib, graphs):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=10, ef=8, seed=0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    step = DeviceBfsRangeStep(dg)
    b = [torch.zeros(V, dtype=torch.uint8, device="cuda") for _ in range(3)]
    i = [torch.zeros(V, dtype=torch.int32, device="cuda") for _ in range(3)]
    c = torch.zeros(4, dtype=torch.int64, device="cuda")
    with pytest.raises(Exception):
        step.init(0, V, V, i[0], i[1], b[0], b[1], i[2], c)  # root out of range
    with pytest.raises(Exception):
        step.expand(5, 3, 0, 1, b[0], b[1], b[2], i[2], i[0], i[1], c)  # lo > hi
    with pytest.raises(Exception):
        step.expand(0, V + 1, 1, 1, b[0], b[1], b[2], i[2], i[0], i[1], c)  # hi > V
    with pytest.raises(Exception):
        step.settle(0, V, 2, 1, i[2], b[2], b[1], i[0], i[1], c)  # direction
    dg.close()


@pytest.mark.parametrize("kind,kw", [("rmat", dict(scale=14, ef=16, seed=3)), ("star", dict(n=20_000, seed=4)),
                                     ("grid", dict(side=80, p=0.01, seed=2)), ("chain", dict(n=600))])
def test_fused_exchange_equals_oracle(torch_cuda, lib, oracle, graphs, kind, kw):
    """ogb_bfs_range_expand_peers / _claim_peers: candidates sent to their
    owner's cand array by atomicMin, owners storing their next bytes into
    every rank's buffer, barriers instead of the all-reduces; each rank a
    thread with its own graph copy, the ranks' buffers local to this GPU."""
    from test_partition_bfs_fused import PeerSet
    torch = torch_cuda
    s, d, _, V = graphs(kind, **kw)
    g = oracle.build(s, d, V, 0)
    E = g["num_edges"]
    gs = _device_graphs(torch, lib, s, d, V, 3)
    try:
        for world in (1, 2, 3):
            ranges = edge_balanced_ranges(g["i_outdeg"], world)
            for root in _roots(g, 2):
                for mode in (2, 0, 1):
                    ps = PeerSet(V, ranges, world, "cuda")
                    outs = run_threads(world, lambda r, dd: bfs_partitioned(DeviceBfsRangeStep(gs[r]), V, E, ranges,
                                                                            r, world, root, "cuda", mode=mode,
                                                                            dist=dd, peers=ps.view(r)))
                    for par, dep, res in outs:
                        check_against_oracle(oracle, g, root, mode, False, host(par, np.int32), host(dep, np.int32),
                                             res)
    finally:
        for dg in gs:
            dg.close()


def _symm_worker(rank, out_path, port):
    import datetime
    import os

    import torch
    import torch.distributed as tdist

    import opengraph_b200 as og
    from conftest import graph_edges
    from oracle.oracle import Oracle
    from opengraph_b200.parallel import SymmetricBfsBuffers
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    tdist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                             device_id=torch.device("cuda", 0))
    try:
        lib = og.load(False)
        lib.quiet(True)
        o = Oracle()
        s, d, _, V = graph_edges("rmat", scale=13, ef=16, seed=2)
        g = o.build(s, d, V, 0)
        dg = lib.device_graph()
        dg.build(dev(torch, s), dev(torch, d), V, 0)
        peers = SymmetricBfsBuffers(V, [(0, V)], "cuda")
        ok = 1
        for root in _roots(g, 2):
            par, dep, res = bfs_partitioned(DeviceBfsRangeStep(dg), V, g["num_edges"], [(0, V)], 0, 1, root, "cuda",
                                            dist=tdist, peers=peers)
            check_against_oracle(o, g, root, 2, False, host(par, np.int32), host(dep, np.int32), res)
        np.save(out_path, np.array([ok]))
        dg.close()
    finally:
        tdist.destroy_process_group()


@pytest.mark.timeout(300)
def test_fused_exchange_through_symmetric_memory(torch_cuda, tmp_path):
    """bfs_partitioned(peers=SymmetricBfsBuffers(...)): cand and the next
    buffers in torch's symmetric memory; one rank of an NCCL group here."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "symm_bfs.npy")
    mp.spawn(_symm_worker, args=(out, port), nprocs=1, join=True)
    assert np.load(out).tolist() == [1]
