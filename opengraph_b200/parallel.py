"""1-D partitioned PageRank pull over several GPUs (one process per GPU).

The reference runs one shared-memory pull loop (pageRank.c:984-1044).  Here
each rank owns a contiguous range of destination vertices -- their
inverse-CSR rows -- chosen so that every range holds about the same number of
in-edges plus vertices (``edge_balanced_ranges``).  Every rank keeps the
whole contrib vector (4 V bytes).  One iteration:

1. the local step: pull over the owned rows against the whole contrib of the
   previous iteration; new ranks and contribs of the owned range, and the
   range's share of the error (sum of |change| / V) and active count;
2. an all-gather of the owned contrib slices (each rank's slice padded to
   the longest), so every rank again holds the whole vector;
3. an all-reduce (sum) of (error, active); the loop stops when no vertex
   changed by epsilon or more, as the reference's does.

At the end the rank slices are all-gathered and divided by V.  The local
step of the product is the library's CUDA kernel (``ogb_pagerank_range_*``),
which sums every row in the same order as the single-GPU pull kernel, so
the ranks do not depend on the partition; the collectives run on whatever
backend the process group has (NCCL between GPUs).  The step object is
passed in, so the partition and exchange logic can also be exercised with
another implementation of the same three calls.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _ptr, _stream


def edge_balanced_ranges(in_degree, parts: int) -> list[tuple[int, int]]:
    """Contiguous vertex ranges [lo, hi) covering [0, V), each holding about
    (E + V) / parts of the work (its in-edges plus one per vertex)."""
    deg = np.asarray(in_degree, dtype=np.int64)
    V = len(deg)
    if parts < 1:
        raise ValueError("parts must be >= 1")
    cum = np.cumsum(deg + 1)
    total = int(cum[-1]) if V else 0
    bounds = [0]
    for k in range(1, parts):
        b = int(np.searchsorted(cum, total * k / parts, side="left")) + 1 if V else 0
        bounds.append(min(V, max(bounds[-1], b)))
    bounds.append(V)
    return [(bounds[k], bounds[k + 1]) for k in range(parts)]


class DeviceRangeStep:
    """The library's CUDA kernels as the local step (device tensors)."""

    def __init__(self, dg, device, stream=None):
        import torch
        self.dg = dg
        self.lib = dg.lib
        self.stream = stream
        self.err = torch.zeros(1, dtype=torch.float64, device=device)
        self.act = torch.zeros(1, dtype=torch.int32, device=device)

    def init(self, ranks, contrib):
        self.lib.check(self.lib.ogb_pagerank_range_init(self.dg.handle, _ptr(ranks), _ptr(contrib),
                                                        _stream(self.stream)), "ogb_pagerank_range_init")

    def step(self, lo, hi, contrib, ranks, contrib_next, epsilon) -> tuple[float, int]:
        """One iteration over [lo, hi); returns the range's (error, active)."""
        self.err.zero_()
        self.act.zero_()
        self.lib.check(self.lib.ogb_pagerank_range_step(self.dg.handle, int(lo), int(hi), _ptr(contrib), _ptr(ranks),
                                                        _ptr(contrib_next), float(epsilon), _ptr(self.err),
                                                        _ptr(self.act), _stream(self.stream)),
                       "ogb_pagerank_range_step")
        return float(self.err.item()), int(self.act.item())

    def finish(self, ranks):
        self.lib.check(self.lib.ogb_pagerank_range_finish(self.dg.handle, _ptr(ranks), _stream(self.stream)),
                       "ogb_pagerank_range_finish")


@dataclass
class PartitionResult:
    iterations: int      # PageRankStats.iterations (index of the stopping iteration)
    executed: int
    error_total: float   # of the last executed iteration
    active: int          # of the last executed iteration
    ranges: list


def pagerank_pull_partitioned(step, V: int, ranges, rank: int, world: int, max_iterations: int, epsilon: float,
                              device, dist=None, group=None):
    """Run the partitioned pull on this rank; returns (the whole normalized
    rank vector on every rank, PartitionResult).  ``dist`` is
    torch.distributed (None for a single process: world must be 1)."""
    import torch
    if world > 1 and dist is None:
        raise ValueError("world > 1 needs torch.distributed")
    lo, hi = ranges[rank]
    maxlen = max(h - l for l, h in ranges)
    ranks = torch.empty(V, dtype=torch.float32, device=device)
    contrib = torch.empty(V, dtype=torch.float32, device=device)
    contrib_next = torch.empty(V, dtype=torch.float32, device=device)
    step.init(ranks, contrib)
    send = torch.zeros(maxlen, dtype=torch.float32, device=device)
    recv = [torch.zeros(maxlen, dtype=torch.float32, device=device) for _ in range(world)]

    def gather_slices(src, dst):
        """dst[l:h] = src[l:h] of every rank's range (all-gather of slices)."""
        if world == 1:
            if dst is not src:
                dst[lo:hi] = src[lo:hi]
            return
        send.zero_()
        send[: hi - lo] = src[lo:hi]
        dist.all_gather(recv, send, group=group)
        for r, (l, h) in enumerate(ranges):
            dst[l:h] = recv[r][: h - l]

    it = executed = 0
    err = 0.0
    act = 0
    for it in range(max_iterations):
        err, act = step.step(lo, hi, contrib, ranks, contrib_next, epsilon)
        if world > 1:
            tot = torch.tensor([err, float(act)], dtype=torch.float64, device=device)
            dist.all_reduce(tot, group=group)
            err, act = float(tot[0].item()), int(round(float(tot[1].item())))
        gather_slices(contrib_next, contrib_next)
        contrib, contrib_next = contrib_next, contrib
        executed = it + 1
        if act == 0:
            break
    else:
        it = max_iterations
    gather_slices(ranks, ranks)
    step.finish(ranks)
    return ranks, PartitionResult(iterations=it, executed=executed, error_total=err, active=act,
                                  ranges=list(ranges))
