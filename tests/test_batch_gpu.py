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


def small_batch(og, n, seed):
    """n seeded RMAT graphs of uneven size (scales 6..11, edge factors 4..16)
    plus a 3-vertex graph without edges; local ids, back to back."""
    rng = np.random.default_rng(seed)
    nv, srcs, dsts = [], [], []
    for i in range(n):
        sc, ef = int(rng.integers(6, 12)), int(rng.integers(4, 17))
        s, d, _ = og.generate_rmat(sc, ef, 1000 + i)
        nv.append(1 << sc)
        srcs.append(s.astype(np.uint32))
        dsts.append(d.astype(np.uint32))
    nv.append(3)
    srcs.append(np.zeros(0, np.uint32))
    dsts.append(np.zeros(0, np.uint32))
    eoff = np.zeros(len(nv) + 1, np.uint64)
    eoff[1:] = np.cumsum([len(x) for x in srcs])
    return nv, eoff, srcs, dsts


def test_batch_equals_single_graphs(torch_cuda, lib, oracle):
    """Every graph of a 24-graph batch: BFS and PageRank equal the
    single-graph path bit for bit, and the oracle (the reference's
    restatement): BFS depths exact, PageRank within 1e-6 L1 of the
    reference's summation order at the executed iteration count."""
    import opengraph_b200 as og
    torch = torch_cuda
    nv, eoff, srcs, dsts = small_batch(og, 24, 0)
    b = og.GraphBatch(lib, nv, eoff, np.concatenate(srcs), np.concatenate(dsts))
    off = b.offsets
    Vt = int(off[-1])
    assert list(np.diff(off)) == nv
    par_t = torch.empty(Vt, dtype=torch.int32, device="cuda")
    dist_t = torch.empty(Vt, dtype=torch.int32, device="cuda")
    rng = np.random.default_rng(3)
    roots = [int(rng.integers(0, x)) for x in nv]
    binfo = b.bfs(roots, par_t, dist_t)
    bpar, bdist = host(par_t, np.int32), host(dist_t)
    ranks_t = torch.empty(Vt, dtype=torch.float32, device="cuda")
    pinfo, per = b.pagerank(ranks_t, max_iterations=100, epsilon=1e-4)
    branks = host(ranks_t, np.float32)
    reached = 0
    for i, V in enumerate(nv):
        lo, hi = int(off[i]), int(off[i + 1])
        dg = lib.device_graph()
        dg.build(dev(torch, srcs[i]), dev(torch, dsts[i]), V, 0)
        p1 = torch.empty(V, dtype=torch.int32, device="cuda")
        d1 = torch.empty(V, dtype=torch.int32, device="cuda")
        dg.bfs(roots[i], p1, d1, mode=2)
        sp, sd = host(p1, np.int32), host(d1)
        assert np.array_equal(bdist[lo:hi], sd), i
        assert np.array_equal(bpar[lo:hi] >= 0, sp >= 0), i
        assert bpar[lo + roots[i]] == roots[i]
        assert np.array_equal(bpar[lo:hi][sp < 0], sp[sp < 0])   # sentinels of unreached vertices
        reached += int((sp >= 0).sum())
        r1 = torch.empty(V, dtype=torch.float32, device="cuda")
        info = dg.pagerank(r1, mode=0, max_iterations=100, epsilon=1e-4)
        assert per[i]["iterations"] == info["iterations"], i
        assert np.array_equal(branks[lo:hi].view(np.uint32), host(r1, np.float32).view(np.uint32)), i
        assert abs(per[i]["error_total"] - info["error_total"]) <= 1e-12 + 1e-9 * abs(info["error_total"]), i
        # against the oracle
        gi = oracle.build(srcs[i], dsts[i], V, 0)
        _, odist, _ = oracle.bfs(gi, roots[i], 2)
        assert np.array_equal(bdist[lo:hi].astype(np.uint32), odist), i
        er, _ = oracle.pagerank(gi, 0, per[i]["executed"], 0.0)
        l1 = float(np.abs(branks[lo:hi].astype(np.float64) - er).sum())
        assert l1 <= 1e-6, (i, l1)
        dg.close()
    assert binfo["reached"] == reached
    # the same call again replays the captured graph
    pinfo2, per2 = b.pagerank(ranks_t, max_iterations=100, epsilon=1e-4)
    assert not pinfo2["captured"] and per2 == per
    assert np.array_equal(host(ranks_t, np.float32).view(np.uint32), branks.view(np.uint32))
    b.close()


def test_batch_autotune_and_bad_input(torch_cuda, lib):
    import opengraph_b200 as og
    torch = torch_cuda
    nv, eoff, srcs, dsts = small_batch(og, 8, 1)
    b = og.GraphBatch(lib, nv, eoff, np.concatenate(srcs), np.concatenate(dsts))
    saved = lib_bins(lib)
    try:
        t = b.autotune()
        assert 0 <= t["best"] < len(t["candidates"])
        best = t["candidates"][t["best"]]
        assert lib_bins(lib)[:2] == best[:2]
        assert best[2] == min(c[2] for c in t["candidates"])
    finally:
        lib.ogb_pagerank_set_bins(saved[0], saved[1])
    b.close()
    with pytest.raises(Exception):   # an id outside its graph
        og.GraphBatch(lib, [4, 4], [0, 1, 2], np.array([0, 5], np.uint32), np.array([1, 1], np.uint32))
    with pytest.raises(Exception):   # a root outside its graph
        b2 = og.GraphBatch(lib, [4], [0, 1], np.array([0], np.uint32), np.array([1], np.uint32))
        p = torch.empty(4, dtype=torch.int32, device="cuda")
        b2.bfs([4], p, p)


def lib_bins(lib):
    import ctypes as C
    w, c, t, k = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    lib.ogb_pagerank_get_bins(C.byref(w), C.byref(c), C.byref(t), C.byref(k))
    return w.value, c.value
