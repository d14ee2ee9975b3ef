"""The multi-GPU bench path on CPU: `bench.py --gpus N` runs N replicas (one
process per GPU), each searching its own seeded roots, and reports the
slowest rank's time with the sum of all ranks' traversed edges.  Two gloo
ranks on the host check that reduction and the per-rank root choice."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        outdeg = (np.arange(5000) * 7919) % 6          # a sixth of the vertices have no out-edges
        roots = bench.rank_roots(outdeg, rank, 32)
        ms, edges = 10.0 + 2.5 * rank, 1000.0 * (rank + 1)
        tot = bench.job_totals(ms, edges, ws, dist, torch.device("cpu"))
        dist.barrier()
        q.put((rank, bench.dist_env(), roots, tot))
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_like_the_bench():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, env, roots, tot = q.get(timeout=120)
        out[rank] = (env, roots, tot)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    outdeg = (np.arange(5000) * 7919) % 6
    for rank in (0, 1):
        env, roots, tot = out[rank]
        assert env == (2, rank, rank)
        assert tot == (12.5, 3000.0)                   # max of the times, sum of the edges
        assert len(set(roots)) == 32 and all(outdeg[r] > 0 for r in roots)
    assert out[0][1] != out[1][1]                      # each replica searches its own roots


def test_single_rank_totals_are_its_own():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_totals(3.0, 42, 1) == (3.0, 42.0)
    outdeg = np.ones(100)
    assert bench.rank_roots(outdeg, 0, 10) == bench.rank_roots(outdeg, 0, 10)
