"""Batched work across ranks (opengraph_b200.parallel.replicas): independent
units split contiguously over the ranks, every rank receiving all result rows
in unit order.  On CPU with a plain function of the unit, as threads
(ThreadDist) and as 2 gloo processes, including fewer units than ranks.  No
GPU."""
import os
import socket

import numpy as np
import pytest

from opengraph_b200.parallel import replicas, split_units
from test_partition_bfs import run_threads


def _rows(units):
    import torch
    return torch.tensor([[u, u * u, -u] for u in units], dtype=torch.int64).reshape(len(units), 3)


def test_split_units_cover_in_order():
    for n in (0, 1, 5, 64, 1000):
        for world in (1, 2, 3, 8):
            parts = [split_units(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("world", [1, 2, 3, 5])
@pytest.mark.parametrize("n", [0, 2, 7, 64])
def test_thread_replicas_gather_all_rows(world, n):
    units = list(range(100, 100 + n))
    want = _rows(units).numpy()
    outs = run_threads(world, lambda r, d: replicas(_rows, units, r, world, dist=d))
    for got in outs:
        assert np.array_equal(got.numpy(), want)


def test_replicas_reject_a_wrong_row_count():
    with pytest.raises(ValueError):
        replicas(lambda us: _rows(us + [0]), [1, 2, 3], 0, 1)


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        got = replicas(_rows, list(range(37)), rank, world, dist=dist)
        np.save(os.path.join(out_dir, f"rows{rank}.npy"), got.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(300)
def test_two_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    want = _rows(list(range(37))).numpy()
    for r in range(2):
        assert np.array_equal(np.load(str(tmp_path / f"rows{r}.npy")), want)
