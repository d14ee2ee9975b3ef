"""The partitioned DO-BFS with the exchange fused into the steps
(bfs_partitioned(..., peers=...)) on CPU: the host protocol -- candidates
sent to their owner's cand array, owners claiming and storing their next
bytes into every rank's buffer, barriers instead of the all-reduces of cand
and next, the two next buffers alternating -- run by thread-ranks over a
PeerSet (every rank's buffers in one process) with a numpy restatement of the
fused steps.  Depths, steps, directions and bottom-up parents must equal the
oracle's single search (BFS.c:476-626), top-down parents the smallest
in-neighbour one level up, as in the unfused exchange.  No GPU."""
import threading

import numpy as np
import pytest

from opengraph_b200.parallel import bfs_partitioned, edge_balanced_ranges, owner_bounds
from test_partition_bfs import CASES, OracleBfsRangeStep, _graph, _roots, check_against_oracle, run_threads

NO_CAND = 0x7F7F7F7F


class PeerSet:
    """world ranks' fused-exchange buffers in one process (test
    infrastructure): rank r's cand and two next buffers, the tensors of every
    rank's addresses, the owner bounds and one barrier for the threads."""

    def __init__(self, V: int, ranges, world: int, device):
        import torch
        self.world = world
        self.cand = [torch.empty(V, dtype=torch.int32, device=device) for _ in range(world)]
        self.next = [[torch.empty(V, dtype=torch.uint8, device=device) for _ in range(2)] for _ in range(world)]
        self.cand_peers = torch.tensor([t.data_ptr() for t in self.cand], dtype=torch.int64, device=device)
        self.next_peers = [torch.tensor([self.next[r][k].data_ptr() for r in range(world)], dtype=torch.int64,
                                        device=device) for k in range(2)]
        self.bounds = torch.tensor(owner_bounds(ranges), dtype=torch.int32, device=device)
        self.bar = threading.Barrier(world, timeout=300)

    def view(self, r: int):
        ps = self

        class View:
            cand = ps.cand[r]
            next = ps.next[r]
            cand_peers = ps.cand_peers
            next_peers = ps.next_peers
            bounds = ps.bounds

            @staticmethod
            def barrier():
                ps.bar.wait()
        return View


class NumpyFusedStep(OracleBfsRangeStep):
    """The fused steps in numpy over a PeerSet (test infrastructure)."""

    def __init__(self, oracle, g, ps: PeerSet, rank: int):
        super().__init__(oracle, g)
        self.ps, self.rank = ps, rank
        self.bounds = np.asarray(ps.bounds.cpu().numpy(), np.int64)

    def expand_peers(self, lo, hi, direction, depth, frontier, visited, nxt, cand_peers, bounds, parents, dist,
                     counts):
        g = self.g
        c = counts.numpy()
        c[:] = 0
        fr, vis = frontier.numpy(), visited.numpy()
        if direction == 0:
            for u in range(lo, hi):
                if not fr[u]:
                    continue
                a = int(g["f_idx"][u])
                for j in range(a, a + int(g["f_outdeg"][u])):
                    w = int(g["f_dst"][j]) & 0x3FFFFFFF
                    if vis[w]:
                        continue
                    o = int(np.searchsorted(self.bounds, w, side="right")) - 1
                    cw = self.ps.cand[o].numpy()
                    if u < cw[w]:
                        cw[w] = u
            return
        nx, par, dep = nxt.numpy(), parents.numpy(), dist.numpy()
        nx[lo:hi] = 0
        for v in range(lo, hi):
            if vis[v]:
                continue
            a = int(g["i_idx"][v])
            for k, j in enumerate(range(a, a + int(g["i_outdeg"][v]))):
                u = int(g["i_dst"][j]) & 0x3FFFFFFF
                if fr[u]:
                    par[v], dep[v], nx[v] = u, depth, 1
                    c[0] += 1
                    c[2] += k + 1
                    break
            else:
                c[2] += int(g["i_outdeg"][v])

    def claim_peers(self, lo, hi, direction, depth, cand, nxt, next_peers, parents, dist, counts):
        k = next(i for i in range(2) if self.ps.next[self.rank][i].data_ptr() == nxt.data_ptr())
        nx = nxt.numpy()
        if direction == 0:
            cd, par, dep, c = cand.numpy(), parents.numpy(), dist.numpy(), counts.numpy()
            od = self.g["f_outdeg"]
            for v in range(lo, hi):
                hit = cd[v] != NO_CAND
                nx[v] = 1 if hit else 0
                if hit:
                    par[v], dep[v] = cd[v], depth
                    c[0] += 1
                    c[1] += max(int(od[v]), 1)
                    cd[v] = NO_CAND
        for r in range(self.ps.world):
            self.ps.next[r][k].numpy()[lo:hi] = nx[lo:hi]

    def settle(self, lo, hi, direction, depth, cand, nxt, visited, parents, dist, counts):
        assert direction == 1  # the fused steps only merge here
        vis = visited.numpy()
        vis |= nxt.numpy()


@pytest.mark.parametrize("kind,kw", CASES)
@pytest.mark.parametrize("world", [1, 2, 3])
def test_fused_exchange_equals_oracle(oracle, kind, kw, world):
    g = _graph(oracle, kind, **kw)
    V, E = g["num_vertices"], g["num_edges"]
    ranges = edge_balanced_ranges(g["i_outdeg"], world)
    for root in _roots(g, 2):
        for mode in (2, 0, 1):
            ps = PeerSet(V, ranges, world, "cpu")
            outs = run_threads(world, lambda r, d: bfs_partitioned(NumpyFusedStep(oracle, g, ps, r), V, E, ranges, r,
                                                                   world, root, "cpu", mode=mode, dist=d,
                                                                   peers=ps.view(r)))
            for par, dep, res in outs:
                check_against_oracle(oracle, g, root, mode, False, par.numpy(), dep.numpy(), res)


def test_fused_exchange_more_ranks_than_vertices(oracle):
    s = np.array([0, 1, 2, 2], np.uint32)
    d = np.array([1, 2, 0, 3], np.uint32)
    g = oracle.build(s, d, 5, 0)
    ranges = edge_balanced_ranges(g["i_outdeg"], 6)
    for root in range(5):
        ps = PeerSet(5, ranges, 6, "cpu")
        outs = run_threads(6, lambda r, dd: bfs_partitioned(NumpyFusedStep(oracle, g, ps, r), 5, g["num_edges"],
                                                            ranges, r, 6, root, "cpu", dist=dd, peers=ps.view(r)))
        for par, dep, res in outs:
            check_against_oracle(oracle, g, root, 2, False, par.numpy(), dep.numpy(), res)


def test_random_graphs_and_cuts_both_exchanges(oracle):
    """Property: on random small graphs (duplicates and self loops
    included) with random owner cut points (empty ranges included), random
    roots and all three modes, the partitioned search with either exchange
    matches the oracle's single search."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=40, deadline=None)
    @given(st.integers(2, 48), st.integers(0, 200), st.integers(1, 4), st.integers(0, 2**31 - 1),
           st.sampled_from([0, 1, 2]), st.booleans())
    def check(V, E, world, seed, mode, fused):
        rng = np.random.default_rng(seed)
        s = rng.integers(0, V, E).astype(np.uint32)
        d = rng.integers(0, V, E).astype(np.uint32)
        g = oracle.build(s, d, V, 0)
        cuts = np.sort(rng.integers(0, V + 1, world - 1))
        bounds = [0] + [int(c) for c in cuts] + [V]
        ranges = [(bounds[r], bounds[r + 1]) for r in range(world)]
        root = int(rng.integers(0, V))
        ps = PeerSet(V, ranges, world, "cpu") if fused else None

        def body(r, dd):
            step = NumpyFusedStep(oracle, g, ps, r) if fused else OracleBfsRangeStep(oracle, g)
            return bfs_partitioned(step, V, g["num_edges"], ranges, r, world, root, "cpu", mode=mode, dist=dd,
                                   peers=ps.view(r) if fused else None)

        for par, dep, res in run_threads(world, body):
            check_against_oracle(oracle, g, root, mode, False, par.numpy(), dep.numpy(), res)

    check()
