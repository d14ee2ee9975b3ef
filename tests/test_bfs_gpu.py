"""GPU parity: BFS (pull, push, direction-optimized) against the oracle.

Distances are compared bit-exactly (unreached vertices keep 0, BFS.c:62);
BFSStats.iteration / processed_nodes and the sequence of TD/BU steps must
match; parents must be valid (root -> root, reached v -> an in-neighbour one
level up, unreached keep the -out_degree / -1 sentinel, BFS.c:58-74), and
bottom-up parents, which the reference chooses deterministically (first
in-neighbour of the frontier in CSR order, BFS.c:736-748), must be equal."""
import numpy as np
import pytest

from test_build_gpu import dev, host

pytestmark = pytest.mark.gpu


def check_parents(g, root, par, dist):
    V = g["num_vertices"]
    outdeg = g["f_outdeg"]
    reached = par >= 0
    assert par[root] == root and dist[root] == 0
    sentinel = np.where(outdeg > 0, -outdeg.astype(np.int64), -1)
    assert np.array_equal(par[~reached].astype(np.int64), sentinel[~reached])
    assert np.all(dist[~reached] == 0)
    v = np.nonzero(reached)[0]
    v = v[v != root]
    p = par[v].astype(np.int64)
    assert np.all((p >= 0) & (p < V))
    assert np.all(dist[p] + 1 == dist[v])
    # (p, v) must be an edge: search v's in-edges (inverse CSR) for p
    idx, deg, nbr = g["i_idx"], g["i_outdeg"], g["i_dst"]
    for vv, pp in zip(v[:20000], p[:20000]):
        row = nbr[idx[vv]: idx[vv] + deg[vv]]
        assert pp in row, (vv, pp)


def roots_of(g, n, seed=0):
    rng = np.random.default_rng(seed)
    cand = np.nonzero(g["f_outdeg"] > 0)[0]
    r = [int(np.argmax(g["f_outdeg"]))]
    r += [int(x) for x in rng.choice(cand, size=min(n - 1, len(cand)), replace=False)]
    return r


CASES = [
    ("rmat", dict(scale=12, ef=16, seed=1)),
    ("rmat", dict(scale=16, ef=16, seed=0)),
    ("uniform", dict(n=40_000, m=200_000, seed=3)),
    ("grid", dict(side=80, p=0.01, seed=2)),
    ("chain", dict(n=3000)),
    ("star", dict(n=20_000, seed=4)),
]


@pytest.mark.parametrize("kind,kw", CASES, ids=[f"{k}-{i}" for i, (k, _) in enumerate(CASES)])
def test_bfs_matches_oracle(torch_cuda, lib, oracle, graphs, kind, kw):
    torch = torch_cuda
    s, d, _, V = graphs(kind, **kw)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    par_t = torch.empty(V, dtype=torch.int32, device="cuda")
    dist_t = torch.empty(V, dtype=torch.int32, device="cuda")
    for root in roots_of(g, 4):
        for mode in (2, 0, 1):
            info = dg.bfs(root, par_t, dist_t, mode=mode)
            par, dist = host(par_t, np.int32), host(dist_t)
            epar, edist, est = oracle.bfs(g, root, mode)
            assert np.array_equal(dist, edist), (root, mode)
            assert info["iteration"] == est["iteration"]
            assert info["processed_nodes"] == est["processed_nodes"]
            assert info["td_steps"] == est["td_steps"] and info["bu_steps"] == est["bu_steps"]
            assert info["reached"] == est["reached"]
            assert info["reached_out_edges"] == est["reached_out_edges"]
            trace = dg.bfs_trace()
            assert [t["direction"] for t in trace] == list(est["dirs"][:len(trace)])
            check_parents(g, root, par, dist)
            if mode == 0:
                assert np.array_equal(par, epar)
    dg.close()


def test_bfs_bad_root(torch_cuda, lib, graphs):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=10, ef=8, seed=0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    par_t = torch.empty(V, dtype=torch.int32, device="cuda")
    dist_t = torch.empty(V, dtype=torch.int32, device="cuda")
    with pytest.raises(Exception):
        dg.bfs(V, par_t, dist_t)
    dg.close()


@pytest.mark.slow
def test_bfs_scale22_properties(torch_cuda, lib, graphs):
    """Full size (RMAT-22, 67M edges): size-independent BFS invariants --
    every edge u->v with u reached has v reached and dist[v] <= dist[u] + 1;
    parents are one level up; the DO run equals the pull-only run."""
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=22, ef=16, seed=0)
    dg = lib.device_graph()
    ts, td = dev(torch, s), dev(torch, d)
    dg.build(ts, td, V, 0)
    par_t = torch.empty(V, dtype=torch.int32, device="cuda")
    dist_t = torch.empty(V, dtype=torch.int32, device="cuda")
    f = dg.view(False)
    outdeg = f.out_degree
    root = int(torch.argmax(outdeg).item())
    dg.bfs(root, par_t, dist_t, mode=2)
    par, dist = par_t.clone(), dist_t.clone()
    reached = par >= 0
    su, dv = ts.long(), td.long()
    ok = ~reached[su] | (reached[dv] & (dist[dv] <= dist[su] + 1))
    assert bool(ok.all())
    v = torch.nonzero(reached).flatten()
    v = v[v != root]
    assert bool((dist[par[v].long()] + 1 == dist[v]).all())
    dg.bfs(root, par_t, dist_t, mode=0)
    assert torch.equal(dist, dist_t)
    dg.close()


def fanout_graph(children: int, per_child: int, seed: int):
    """Root 0 -> `children` vertices -> `per_child` grandchildren each (some
    shared, so claims race), plus edges back to the root: the second
    top-down level expands a list of exactly `children` entries."""
    rng = np.random.default_rng(seed)
    kids = np.arange(1, children + 1, dtype=np.uint32)
    V = 1 + children + children * per_child // 2
    gkids = rng.integers(children + 1, V, size=(children, per_child)).astype(np.uint32)
    s = np.concatenate([np.zeros(children, np.uint32), np.repeat(kids, per_child), gkids[:, 0]])
    d = np.concatenate([kids, gkids.reshape(-1), np.zeros(children, np.uint32)])
    return s, d, int(V)


@pytest.mark.parametrize("children", [1000, 1024, 1025, 3000, 4096, 4097, 6000])
def test_bfs_top_down_list_sizes(torch_cuda, lib, oracle, children):
    """Top-down steps over lists of at most 1024 entries (one phase, every
    CTA scans the list), 1025..4096 (one phase, tile owners scan it) and
    more (two phases, chained scan): depths, counts and parents as the
    oracle, in push-only and direction-optimized modes."""
    torch = torch_cuda
    s, d, V = fanout_graph(children, 5, children)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    par_t = torch.empty(V, dtype=torch.int32, device="cuda")
    dist_t = torch.empty(V, dtype=torch.int32, device="cuda")
    for mode in (1, 2):
        info = dg.bfs(0, par_t, dist_t, mode=mode)
        par, dist = host(par_t, np.int32), host(dist_t)
        _, edist, est = oracle.bfs(g, 0, mode)
        assert np.array_equal(dist, edist), mode
        assert info["iteration"] == est["iteration"] and info["reached"] == est["reached"]
        assert [t["direction"] for t in dg.bfs_trace()] == list(est["dirs"][:info["levels"]])
        check_parents(g, 0, par, dist)
    dg.close()
