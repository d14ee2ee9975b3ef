"""GPU parity: multi-source BFS (up to 64 roots as bit-lanes).

Every lane must equal a single-root BFS of the oracle bit for bit: the depth
of each reached vertex equals the oracle's distance, and exactly the vertices
the oracle reaches (parent >= 0) are reached (others read 0xFFFF).  Covers
64 lanes, a partial batch, duplicate roots, roots without out-edges and a
high-diameter grid."""
import numpy as np
import pytest

from test_build_gpu import dev, host

pytestmark = pytest.mark.gpu

UNREACHED = 0xFFFF

CASES = [
    ("rmat", dict(scale=12, ef=16, seed=1)),
    ("rmat", dict(scale=15, ef=16, seed=0)),
    ("uniform", dict(n=40_000, m=200_000, seed=3)),
    ("grid", dict(side=80, p=0.01, seed=2)),
    ("star", dict(n=20_000, seed=4)),
]


def lane_roots(g, n, seed):
    rng = np.random.default_rng(seed)
    V = g["num_vertices"]
    cand = np.nonzero(g["f_outdeg"] > 0)[0]
    roots = [int(x) for x in rng.choice(cand, size=min(n, len(cand)), replace=False)]
    if n >= 4 and len(roots) >= 4:
        roots[1] = roots[0]                                   # duplicate root: two lanes, one vertex
        zero = np.nonzero(g["f_outdeg"] == 0)[0]
        if len(zero):
            roots[2] = int(zero[0])                           # a root without out-edges
        roots[3] = V - 1
    return roots


def check_lanes(oracle, g, roots, depths):
    for lane, r in enumerate(roots):
        par, dist, _ = oracle.bfs(g, r, 2)
        got = depths[:, lane].astype(np.int64)
        reached = par >= 0
        assert np.array_equal(got != UNREACHED, reached), (lane, r)
        assert np.array_equal(got[reached], dist[reached].astype(np.int64)), (lane, r)


@pytest.mark.parametrize("kind,kw", CASES, ids=[f"{k}-{i}" for i, (k, _) in enumerate(CASES)])
def test_msbfs_lanes_equal_single_bfs(torch_cuda, lib, oracle, graphs, kind, kw):
    torch = torch_cuda
    s, d, _, V = graphs(kind, **kw)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    depth_t = torch.empty(V * 64, dtype=torch.int16, device="cuda")
    for n, seed in ((64, 0), (7, 1)):
        roots = lane_roots(g, n, seed)
        info = dg.msbfs(roots, depth_t)
        depths = host(depth_t, np.int16).view(np.uint16).reshape(V, 64)
        check_lanes(oracle, g, roots, depths)
        assert np.all(depths[:, len(roots):] == UNREACHED)
        assert info["reached_pairs"] == int((depths[:, :len(roots)] != UNREACHED).sum())
        assert info["push_levels"] + info["pull_levels"] == info["levels"]
    dg.close()


def test_msbfs_rejects_bad_roots(torch_cuda, lib, graphs):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=10, ef=8, seed=0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    depth_t = torch.empty(V * 64, dtype=torch.int16, device="cuda")
    with pytest.raises(Exception):
        dg.msbfs([V], depth_t)
    with pytest.raises(Exception):
        dg.msbfs(list(range(65)), depth_t)
    with pytest.raises(Exception):
        dg.msbfs([], depth_t)
    dg.close()


PPR_CASES = [
    ("rmat", dict(scale=12, ef=16, seed=1)),
    ("uniform", dict(n=20_000, m=100_000, seed=3)),
    ("grid", dict(side=60, p=0.01, seed=2)),
    ("star", dict(n=5_000, seed=4)),
]
PPR_L1_TOL = 1e-5  # per seed vector (mass <= 1): fp32 sums vs the FP64 restatement


@pytest.mark.parametrize("kind,kw", PPR_CASES, ids=[f"{k}-{i}" for i, (k, _) in enumerate(PPR_CASES)])
def test_ppr_vs_fp64(torch_cuda, lib, oracle, graphs, kind, kw):
    torch = torch_cuda
    s, d, _, V = graphs(kind, **kw)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    ranks_t = torch.empty(V * 32, dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(7)
    for n in (32, 5):
        seeds = [int(x) for x in rng.choice(V, size=n, replace=False)]
        if n == 32:
            seeds[1] = seeds[0]                                  # duplicate seed: identical vectors
            seeds[2] = int(np.argmax(g["i_outdeg"]))             # the in-hub
        info = dg.ppr(seeds, ranks_t, max_iterations=20, epsilon=0.0)
        got = host(ranks_t, np.float32).reshape(V, 32)[:, :n].astype(np.float64)
        want, hist = oracle.ppr_f64(g, seeds, 20)
        l1 = np.abs(got - want).sum(axis=0)
        assert np.all(l1 <= PPR_L1_TOL), (n, l1.max())
        assert np.allclose(info["err_last"], hist[-1], rtol=1e-4, atol=1e-7)
        assert info["executed"] == 20 and not info["converged"]
        if n == 32:
            assert np.array_equal(got[:, 0], got[:, 1])
    dg.close()


def test_ppr_stops_on_epsilon(torch_cuda, lib, oracle, graphs):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=11, ef=8, seed=2)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    seeds = list(range(0, 64, 2))
    info = dg.ppr(seeds, None, max_iterations=200, epsilon=1e-6)
    assert info["converged"] and info["executed"] < 200
    _, hist = oracle.ppr_f64(g, seeds, info["executed"])
    # the run stopped at the first iteration whose every vector changed by < 1e-6
    assert hist[-1].max() < 1.5e-6
    assert hist[-2].max() >= 0.5e-6
    with pytest.raises(Exception):
        dg.ppr(list(range(33)), None)
    with pytest.raises(Exception):
        dg.ppr([V], None)
    dg.close()
