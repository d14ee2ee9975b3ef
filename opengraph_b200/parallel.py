"""Work over several GPUs (one process per GPU): the graph build from
edge-list shards, the 1-D partitioned PageRank pull and direction-optimizing
BFS, and replicas of the batched work.

PageRank pull
-------------
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
another implementation of the same three calls.  With ``fused=True`` the
all-gather moves into the step: the next-contrib buffers live in symmetric
memory (``PeerContribs``) and the range kernel stores each contrib it
computes into every rank's copy, so an iteration ends with a barrier.

Batched work
------------
Multi-source BFS roots, personalized-PageRank seeds and small graphs are
independent units: ``replicas`` gives each rank a contiguous share, runs the
library's batched kernels on it against its own copy of the graph, and
all-gathers the result rows in unit order (``msbfs_replicas``,
``ppr_replicas``).  There is no exchange inside the work.

Graph build
-----------
``exchange_edges`` turns each rank's shard of the edge list (the shards in
rank order form the whole list) into the edges its graph needs: every edge
goes to the owner of its source and to the owner of its destination (the
library's stable split, ``ogb_partition_edges``, then an all-to-all).  The
graph a rank builds from them (``partitioned_device_graph``) holds, for each
vertex it owns, the out-row and in-row of the whole graph in the same order,
which is all the partitioned PageRank and BFS steps read; each edge is
stored on at most two ranks.  With the whole graph on every rank instead,
the same steps give the same results.

Direction-optimizing BFS
------------------------
The reference runs one shared-memory loop (BFS.c:476-626).  Here each rank
owns a contiguous vertex range (edge-balanced by in-degree, as above): their
parents and depths, their out-rows for top-down steps and their in-rows for
bottom-up steps.  Every rank keeps the frontier and the visited set as one
byte per vertex over all V.  One step:

1. expand (the library's kernels): top-down, every unvisited out-neighbour
   w of an owned frontier vertex u gets cand[w] = min(cand[w], u);
   bottom-up, each owned unvisited vertex takes its first in-neighbour in
   the frontier as parent and sets its next byte;
2. the exchange: top-down a min all-reduce of cand (4 V bytes), bottom-up a
   max all-reduce of the next bytes (V bytes);
3. settle: top-down, the vertices with a cand form the next frontier, and
   each owner gives its own their parent (cand: the smallest frontier
   in-neighbour) and depth and counts them and the reference's mf; then
   visited |= next;
4. a sum all-reduce of the step's counts, from which every rank takes the
   same direction decision (the switch of BFS.c:546-587: mu, mf, nf with
   alpha 15 and beta 18, in the reference's u32 arithmetic).

With ``peers`` (SymmetricBfsBuffers) the exchange is fused into the steps:
a top-down expand sends each candidate to its owner's cand array (remote
atomicMin over NVLink), the owner claims and stores its next bytes into
every rank's buffer, and barriers replace the two all-reduces of cand and
next; only the four counters are still all-reduced.

Depths, the step count and every step's direction equal the single-GPU
search's (and the reference's); bottom-up parents are the reference's too
(the first frontier in-neighbour in CSR order), top-down parents the
smallest frontier in-neighbour (the reference's are whichever frontier
vertex wins a race); neither depends on the partition.  At the end the owned
slices of parents and depths are all-gathered.
"""
from __future__ import annotations

import ctypes as C
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

    def step(self, lo, hi, contrib, ranks, contrib_next, epsilon, peers=None) -> tuple[float, int]:
        """One iteration over [lo, hi); returns the range's (error, active).
        peers: a device int64 tensor of buffer addresses that also receive
        contrib_next on [lo, hi) (the fused exchange)."""
        self.err.zero_()
        self.act.zero_()
        if peers is None:
            self.lib.check(self.lib.ogb_pagerank_range_step(self.dg.handle, int(lo), int(hi), _ptr(contrib),
                                                            _ptr(ranks), _ptr(contrib_next), float(epsilon),
                                                            _ptr(self.err), _ptr(self.act), _stream(self.stream)),
                           "ogb_pagerank_range_step")
        else:
            self.lib.check(self.lib.ogb_pagerank_range_step_peers(self.dg.handle, int(lo), int(hi), _ptr(contrib),
                                                                  _ptr(ranks), _ptr(contrib_next), _ptr(peers),
                                                                  int(peers.numel()), float(epsilon), _ptr(self.err),
                                                                  _ptr(self.act), _stream(self.stream)),
                           "ogb_pagerank_range_step_peers")
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


class PeerContribs:
    """The fused exchange of the partitioned pull: the two next-contrib
    buffers in symmetric memory (torch.distributed._symmetric_memory), mapped
    on every rank, so a range step stores each owned contrib into every
    rank's copy over NVLink (``ogb_pagerank_range_step_peers``) instead of an
    all-gather after it."""

    def __init__(self, V: int, device, group=None):
        import torch
        import torch.distributed as tdist
        import torch.distributed._symmetric_memory as symm
        g = group if group is not None else tdist.group.WORLD
        self.bufs = [symm.empty(V, dtype=torch.float32, device=device) for _ in range(2)]
        self.handles = [symm.rendezvous(b, g.group_name) for b in self.bufs]
        self.peers = [torch.tensor([int(x) for x in h.buffer_ptrs], dtype=torch.int64, device=device)
                      for h in self.handles]

    def barrier(self, k: int):
        self.handles[k].barrier()


def pagerank_pull_partitioned(step, V: int, ranges, rank: int, world: int, max_iterations: int, epsilon: float,
                              device, dist=None, group=None, fused: bool = False):
    """Run the partitioned pull on this rank; returns (the whole normalized
    rank vector on every rank, PartitionResult).  ``dist`` is
    torch.distributed (None for a single process: world must be 1).  fused:
    the contrib exchange inside the range step (peer stores into symmetric
    memory, then a barrier) instead of an all-gather after it; GPUs with a
    process group only."""
    import torch
    if world > 1 and dist is None:
        raise ValueError("world > 1 needs torch.distributed")
    lo, hi = ranges[rank]
    maxlen = max(h - l for l, h in ranges)
    ranks = torch.empty(V, dtype=torch.float32, device=device)
    peer = PeerContribs(V, device, group) if fused else None
    if peer is not None:
        contrib, contrib_next = peer.bufs
        which = 1  # the buffer contrib_next is
    else:
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

    # the owners' contribs: with a partitioned graph only they have whole out-degrees
    gather_slices(contrib, contrib)
    it = executed = 0
    err = 0.0
    act = 0
    for it in range(max_iterations):
        if peer is not None:
            err, act = step.step(lo, hi, contrib, ranks, contrib_next, epsilon, peers=peer.peers[which])
        else:
            err, act = step.step(lo, hi, contrib, ranks, contrib_next, epsilon)
        if world > 1:
            tot = torch.tensor([err, float(act)], dtype=torch.float64, device=device)
            dist.all_reduce(tot, group=group)
            err, act = float(tot[0].item()), int(round(float(tot[1].item())))
        if peer is not None:
            peer.barrier(which)  # every rank's stores into every copy are done
            which ^= 1
        else:
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


class DeviceBfsRangeStep:
    """The library's CUDA kernels as one rank's BFS step (device tensors)."""

    def __init__(self, dg, stream=None):
        self.dg = dg
        self.lib = dg.lib
        self.stream = stream

    def init(self, lo, hi, root, parents, dist, frontier, visited, cand, counts):
        self.lib.check(self.lib.ogb_bfs_range_init(self.dg.handle, int(lo), int(hi), int(root), _ptr(parents),
                                                   _ptr(dist), _ptr(frontier), _ptr(visited), _ptr(cand),
                                                   _ptr(counts), _stream(self.stream)), "ogb_bfs_range_init")

    def expand(self, lo, hi, direction, depth, frontier, visited, nxt, cand, parents, dist, counts):
        self.lib.check(self.lib.ogb_bfs_range_expand(self.dg.handle, int(lo), int(hi), int(direction), int(depth),
                                                     _ptr(frontier), _ptr(visited), _ptr(nxt), _ptr(cand),
                                                     _ptr(parents), _ptr(dist), _ptr(counts), _stream(self.stream)),
                       "ogb_bfs_range_expand")

    def settle(self, lo, hi, direction, depth, cand, nxt, visited, parents, dist, counts):
        self.lib.check(self.lib.ogb_bfs_range_settle(self.dg.handle, int(lo), int(hi), int(direction), int(depth),
                                                     _ptr(cand), _ptr(nxt), _ptr(visited), _ptr(parents),
                                                     _ptr(dist), _ptr(counts), _stream(self.stream)),
                       "ogb_bfs_range_settle")

    def expand_peers(self, lo, hi, direction, depth, frontier, visited, nxt, cand_peers, bounds, parents, dist,
                     counts):
        self.lib.check(self.lib.ogb_bfs_range_expand_peers(self.dg.handle, int(lo), int(hi), int(direction),
                                                           int(depth), _ptr(frontier), _ptr(visited), _ptr(nxt),
                                                           _ptr(cand_peers), _ptr(bounds), int(bounds.numel()) - 1,
                                                           _ptr(parents), _ptr(dist), _ptr(counts),
                                                           _stream(self.stream)), "ogb_bfs_range_expand_peers")

    def claim_peers(self, lo, hi, direction, depth, cand, nxt, next_peers, parents, dist, counts):
        self.lib.check(self.lib.ogb_bfs_range_claim_peers(self.dg.handle, int(lo), int(hi), int(direction),
                                                          int(depth), _ptr(cand), _ptr(nxt), _ptr(next_peers),
                                                          int(next_peers.numel()), _ptr(parents), _ptr(dist),
                                                          _ptr(counts), _stream(self.stream)),
                       "ogb_bfs_range_claim_peers")


class SymmetricBfsBuffers:
    """The fused exchange of the partitioned BFS: this rank's cand array and
    two alternating next buffers in symmetric memory
    (torch.distributed._symmetric_memory), every rank's addresses of them,
    and the owner bounds, as ``bfs_partitioned(..., peers=...)`` takes them."""

    def __init__(self, V: int, ranges, device, group=None):
        import torch
        import torch.distributed as tdist
        import torch.distributed._symmetric_memory as symm
        g = group if group is not None else tdist.group.WORLD
        self.cand = symm.empty(V, dtype=torch.int32, device=device)
        self.next = [symm.empty(V, dtype=torch.uint8, device=device) for _ in range(2)]
        bufs = [self.cand, self.next[0], self.next[1]]
        self.handles = [symm.rendezvous(b, g.group_name) for b in bufs]
        ptrs = [torch.tensor([int(x) for x in h.buffer_ptrs], dtype=torch.int64, device=device) for h in self.handles]
        self.cand_peers, self.next_peers = ptrs[0], ptrs[1:]
        self.bounds = torch.tensor(owner_bounds(ranges), dtype=torch.int32, device=device)

    def barrier(self):
        self.handles[0].barrier()


@dataclass
class BfsPartitionResult:
    iteration: int        # BFSStats.iteration: steps + 1
    processed_nodes: int  # BFSStats.processed_nodes: vertices reached, root included
    td_steps: int
    bu_steps: int
    directions: list      # per step: 0 top-down, 1 bottom-up
    edges_examined: int   # in-edges read by the bottom-up steps, all ranks
    ranges: list


_U32 = 0xFFFFFFFF


def bfs_partitioned(step, V: int, E: int, ranges, rank: int, world: int, root: int, device, mode: int = 2,
                    bu_entry_nf_frontier: bool = False, dist=None, group=None, peers=None):
    """Run the partitioned BFS on this rank; returns (parents, depths as
    int32 tensors of V, the whole vectors on every rank; BfsPartitionResult).
    mode 0 bottom-up only, 1 top-down only, 2 direction-optimizing;
    bu_entry_nf_frontier starts a bottom-up run with nf = the frontier size
    (the bitmap variant) instead of 0.  ``dist`` is torch.distributed (None
    for a single process: world must be 1).  peers: the fused exchange's
    buffers (SymmetricBfsBuffers: cand, next[2], cand_peers, next_peers[2],
    bounds, barrier()); the steps then send candidates and next bytes
    straight to the ranks that need them, with barriers instead of the
    all-reduces of cand and next."""
    import torch
    if world > 1 and dist is None:
        raise ValueError("world > 1 needs torch.distributed")
    if mode not in (0, 1, 2):
        raise ValueError("mode: 0 bottom-up, 1 top-down, 2 direction-optimizing")
    if not 0 <= root < V:
        raise ValueError(f"root {root} out of range (V={V})")
    lo, hi = ranges[rank]
    parents = torch.empty(V, dtype=torch.int32, device=device)
    depths = torch.empty(V, dtype=torch.int32, device=device)
    visited = torch.empty(V, dtype=torch.uint8, device=device)
    counts = torch.zeros(4, dtype=torch.int64, device=device)
    which = 0  # fused exchange: the next buffer that holds the frontier
    if peers is None:
        frontier = torch.empty(V, dtype=torch.uint8, device=device)
        nxt = torch.empty(V, dtype=torch.uint8, device=device)
        cand = torch.empty(V, dtype=torch.int32, device=device)
    else:
        frontier, nxt, cand = peers.next[0], peers.next[1], peers.cand
    step.init(lo, hi, root, parents, depths, frontier, visited, cand, counts)
    if peers is not None:
        peers.barrier()  # every rank's cand and frontier set before any rank writes into them
    if world > 1:
        dist.all_reduce(counts, group=group)  # the root's owner holds its out-degree
    mf = int(counts[1].item()) & _U32
    mu = E & _U32
    alpha, beta = 15, 18
    qn, nf = 1, 0
    iteration = processed = 1
    td = bu = 0
    dirs = []
    examined = 0

    def run(direction):
        nonlocal frontier, nxt, examined, which
        depth = len(dirs) + 1
        if peers is None:
            step.expand(lo, hi, direction, depth, frontier, visited, nxt, cand, parents, depths, counts)
            if world > 1:
                if direction == 0:
                    dist.all_reduce(cand, op=dist.ReduceOp.MIN, group=group)
                else:
                    dist.all_reduce(nxt, op=dist.ReduceOp.MAX, group=group)
            step.settle(lo, hi, direction, depth, cand, nxt, visited, parents, depths, counts)
        else:
            step.expand_peers(lo, hi, direction, depth, frontier, visited, nxt, peers.cand_peers, peers.bounds,
                              parents, depths, counts)
            if direction == 0:
                peers.barrier()  # every candidate is in its owner's cand
            step.claim_peers(lo, hi, direction, depth, cand, nxt, peers.next_peers[which ^ 1], parents, depths,
                             counts)
            peers.barrier()  # every owner's next bytes are in every rank's buffer
            step.settle(lo, hi, 1, depth, cand, nxt, visited, parents, depths, counts)  # visited |= next
            which ^= 1
        if world > 1:
            dist.all_reduce(counts, group=group)
        c = [int(x) for x in counts.tolist()]
        if c[3]:
            raise RuntimeError("partitioned bfs: a step queue overflowed")
        frontier, nxt = nxt, frontier
        dirs.append(direction)
        examined += c[2]
        return c

    while qn > 0:
        if mode == 0 or (mode == 2 and mf > mu // alpha):
            nf = qn if bu_entry_nf_frontier else 0
            while True:
                nf_prev = nf
                nf = run(1)[0]
                iteration += 1
                processed += nf
                bu += 1
                if not (nf > 0 if mode == 0 else (nf > nf_prev or nf > V // beta)):
                    break
            qn = nf
            mf = 1
        else:
            mu = (mu - mf) & _U32
            c = run(0)
            mf = c[1] & _U32
            qn = c[0]
            iteration += 1
            processed += qn
            td += 1

    if world > 1:
        maxlen = max(h - l for l, h in ranges)
        for t in (parents, depths):
            send = torch.zeros(maxlen, dtype=t.dtype, device=device)
            send[: hi - lo] = t[lo:hi]
            recv = [torch.zeros(maxlen, dtype=t.dtype, device=device) for _ in range(world)]
            dist.all_gather(recv, send, group=group)
            for r, (l, h) in enumerate(ranges):
                t[l:h] = recv[r][: h - l]
    return parents, depths, BfsPartitionResult(iteration=iteration, processed_nodes=processed, td_steps=td,
                                               bu_steps=bu, directions=dirs, edges_examined=examined,
                                               ranges=list(ranges))


def shard_ranges(dst, V: int, world: int, dist=None, group=None) -> list[tuple[int, int]]:
    """edge_balanced_ranges of the whole graph's in-degrees, from this rank's
    shard of destination ids (a V-entry count summed over the ranks).
    Duplicate edges and self loops count as they stand."""
    import torch
    deg = torch.bincount(dst.long(), minlength=V)[:V].to(torch.int64)
    if world > 1:
        dist.all_reduce(deg, group=group)
    return edge_balanced_ranges(deg.cpu().numpy(), world)


def owner_bounds(ranges) -> list[int]:
    """[lo_0, lo_1, ..., hi_last]: the ranges as the partition kernel takes them."""
    return [int(lo) for lo, _ in ranges] + [int(ranges[-1][1])]


class DeviceEdgeSplit:
    """The library's stable split of an edge shard by owner (device tensors)."""

    def __init__(self, lib, stream=None):
        self.lib = lib
        self.stream = stream

    def split(self, src, dst, w, bounds):
        """Returns (out_src, out_dst, out_w or None, counts per owner)."""
        import torch
        E = int(src.numel())
        n = len(bounds) - 1
        cap = max(2 * E, 1)
        out_src = torch.empty(cap, dtype=src.dtype, device=src.device)
        out_dst = torch.empty(cap, dtype=dst.dtype, device=dst.device)
        out_w = torch.empty(cap, dtype=torch.float32, device=src.device) if w is not None else None
        b = (C.c_uint32 * (n + 1))(*bounds)
        cnt = (C.c_uint32 * n)()
        self.lib.check(self.lib.ogb_partition_edges(_ptr(src), _ptr(dst), _ptr(w), E, b, n, _ptr(out_src),
                                                    _ptr(out_dst), _ptr(out_w), cnt, _stream(self.stream)),
                       "ogb_partition_edges")
        return out_src, out_dst, out_w, [int(x) for x in cnt]


def exchange_edges(split, src, dst, w, ranges, rank: int, world: int, dist=None, group=None):
    """This rank's shard (src, dst[, w]) in, the edges this rank's graph needs
    out: (src, dst, w or None, total edges of all shards).  ``split`` is a
    DeviceEdgeSplit (or another implementation of ``split``); the received
    segments are in sender order."""
    import torch
    if world > 1 and dist is None:
        raise ValueError("world > 1 needs torch.distributed")
    out_src, out_dst, out_w, counts = split.split(src, dst, w, owner_bounds(ranges))
    n_total = torch.tensor([int(src.numel())], dtype=torch.int64, device=src.device)
    if world == 1:
        n = counts[0]
        return out_src[:n], out_dst[:n], (out_w[:n] if out_w is not None else None), int(n_total.item())
    send_n = torch.tensor(counts, dtype=torch.int64, device=src.device)
    recv_n = torch.empty(world, dtype=torch.int64, device=src.device)
    dist.all_to_all_single(recv_n, send_n, group=group)
    rc = [int(x) for x in recv_n.tolist()]
    sent = sum(counts)

    def a2a(t):
        x = t[:sent].contiguous()
        if x.dtype == torch.uint32:  # 32-bit ids cross as int32 (not every backend takes uint32)
            x = x.view(torch.int32)
        r = torch.empty(sum(rc), dtype=x.dtype, device=t.device)
        dist.all_to_all_single(r, x, output_split_sizes=rc, input_split_sizes=counts, group=group)
        return r.view(t.dtype)

    rs, rd = a2a(out_src), a2a(out_dst)
    rw = a2a(out_w) if out_w is not None else None
    dist.all_reduce(n_total, group=group)
    return rs, rd, rw, int(n_total.item())


def partitioned_device_graph(lib, src, dst, w, V: int, ranges, rank: int, world: int, sort_type: int = 0,
                             dist=None, group=None, stream=None):
    """Build this rank's part of a graph split by ``ranges`` from this rank's
    shard of the edge list (device tensors).  Returns (DeviceGraph, total
    edges E of the whole graph: the DO-BFS switch's mu)."""
    s, d, ww, E = exchange_edges(DeviceEdgeSplit(lib, stream), src, dst, w, ranges, rank, world, dist, group)
    dg = lib.device_graph()
    dg.build(s, d, V, sort_type, weight=ww, stream=stream)
    return dg, E


def split_units(n: int, rank: int, world: int) -> tuple[int, int]:
    """This rank's contiguous share [a, b) of n independent units."""
    return n * rank // world, n * (rank + 1) // world


def replicas(run, units, rank: int, world: int, dist=None, group=None):
    """Independent units (roots, seeds, graphs) split across the ranks: this
    rank runs ``run(its units)``, which returns a tensor with one row per
    unit; every rank gets the rows of all units, in unit order (an all-gather
    of the shares, padded to the largest)."""
    import torch
    if world > 1 and dist is None:
        raise ValueError("world > 1 needs torch.distributed")
    units = list(units)
    n = len(units)
    a, b = split_units(n, rank, world)
    local = run(units[a:b])
    if local.shape[0] != b - a:
        raise ValueError(f"run returned {local.shape[0]} rows for {b - a} units")
    if world == 1:
        return local
    sizes = [split_units(n, r, world)[1] - split_units(n, r, world)[0] for r in range(world)]
    pad = torch.zeros((max(sizes),) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: b - a] = local
    recv = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(recv, pad, group=group)
    return torch.cat([recv[r][: sizes[r]] for r in range(world)])


def msbfs_replicas(dg, roots, rank: int, world: int, dist=None, group=None, stream=None):
    """Depths of many single-source searches (one row per root, V uint16
    entries, 0xFFFF unreached), the roots split across the ranks and run 64
    at a time by the library's multi-source BFS (``ogb_msbfs``) on each rank's
    copy of the graph."""
    import torch

    def run(rs):
        V = dg.view(False).num_vertices
        out = torch.empty((len(rs), V), dtype=torch.int16, device="cuda")
        depths = torch.empty(V * 64, dtype=torch.int16, device="cuda")
        for i in range(0, len(rs), 64):
            chunk = rs[i: i + 64]
            dg.msbfs(chunk, depths, stream=stream)
            out[i: i + len(chunk)] = depths.view(V, 64)[:, : len(chunk)].t()
        return out
    return replicas(run, roots, rank, world, dist, group)


def ppr_replicas(dg, seeds, rank: int, world: int, max_iterations: int = 20, epsilon: float = 0.0, dist=None,
                 group=None, stream=None):
    """Personalized PageRank vectors (one row per seed, V float32), the seeds
    split across the ranks and run 32 at a time by the library's batched PPR
    (``ogb_ppr``) on each rank's copy of the graph."""
    import torch

    def run(ss):
        V = dg.view(False).num_vertices
        out = torch.empty((len(ss), V), dtype=torch.float32, device="cuda")
        ranks = torch.empty(V * 32, dtype=torch.float32, device="cuda")
        for i in range(0, len(ss), 32):
            chunk = ss[i: i + 32]
            dg.ppr(chunk, ranks, max_iterations=max_iterations, epsilon=epsilon, stream=stream)
            out[i: i + len(chunk)] = ranks.view(V, 32)[:, : len(chunk)].t()
        return out
    return replicas(run, seeds, rank, world, dist, group)
