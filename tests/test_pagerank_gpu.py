"""GPU parity: PageRank pull and push against the oracle's fp32 restatement
of pageRank.c:939-1186 (itself pinned bit-exactly to the reference's pull).

Tolerance: normalized ranks within 1e-6 L1 of the oracle at the same
iteration count (the in-degree > 32 vertices are summed in a different order
than the reference's sequential loop).  Vertices of in-degree <= 32 are summed
sequentially in CSR order and must match bit-exactly in pull mode as long as
the inputs do; the error against an FP64 oracle is reported."""
import numpy as np
import pytest

from test_build_gpu import dev, host

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


CASES = [
    ("rmat", dict(scale=12, ef=16, seed=1)),
    ("rmat", dict(scale=16, ef=16, seed=0)),
    ("uniform", dict(n=40_000, m=200_000, seed=3)),
    ("grid", dict(side=80, p=0.01, seed=2)),
    ("star", dict(n=20_000, seed=4)),
]


@pytest.mark.parametrize("kind,kw", CASES, ids=[f"{k}-{i}" for i, (k, _) in enumerate(CASES)])
@pytest.mark.parametrize("mode", [0, 1])
def test_pagerank_matches_oracle(torch_cuda, lib, oracle, graphs, kind, kw, mode):
    torch = torch_cuda
    s, d, _, V = graphs(kind, **kw)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    ranks_t = torch.empty(V, dtype=torch.float32, device="cuda")
    # fixed iteration count (epsilon 0 never stops early) and the default stop rule
    for iters, eps in ((20, 0.0), (100, 1e-4)):
        info = dg.pagerank(ranks_t, mode=mode, max_iterations=iters, epsilon=eps)
        ranks = host(ranks_t, np.float32)
        er, ei = oracle.pagerank(g, mode, iters, eps)
        assert info["iterations"] == ei["iterations"], (info, ei["iterations"])
        l1 = float(np.abs(ranks.astype(np.float64) - er).sum())
        assert l1 <= L1_TOL, l1
        assert abs(info["error_total"] - ei["error_total"]) <= 1e-6 * max(1.0, ei["error_total"]) + 1e-9
        errs, act = dg.pagerank_history()
        assert len(errs) == ei["executed"]
    if mode == 0:
        # in-degree <= 32 vertices: identical summation order -> identical ranks
        # after one iteration
        dg.pagerank(ranks_t, mode=0, max_iterations=1, epsilon=0.0)
        er, _ = oracle.pagerank(g, 0, 1, 0.0)
        small = g["i_outdeg"] <= 32
        assert np.array_equal(host(ranks_t, np.float32)[small], er[small])
    dg.close()


def test_pagerank_fp64_error_stated(torch_cuda, lib, oracle, graphs):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=14, ef=16, seed=2)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    ranks_t = torch.empty(V, dtype=torch.float32, device="cuda")
    dg.pagerank(ranks_t, mode=0, max_iterations=30, epsilon=0.0)
    r64 = oracle.pagerank_f64(g, 30)
    l1 = float(np.abs(host(ranks_t, np.float32).astype(np.float64) - r64).sum())
    print(f"fp32 GPU vs fp64 oracle L1 after 30 iterations: {l1:.3e}")
    assert l1 < 1e-5
    dg.close()


def test_pagerank_init_vector(torch_cuda, lib, oracle, graphs):
    torch = torch_cuda
    s, d, _, V = graphs("rmat", scale=12, ef=16, seed=1)
    g = oracle.build(s, d, V, 0)
    dg = lib.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0)
    init = np.random.default_rng(0).uniform(0.1, 2.0, V).astype(np.float32)
    ranks_t = torch.empty(V, dtype=torch.float32, device="cuda")
    info = dg.pagerank(ranks_t, mode=0, max_iterations=50, epsilon=1e-6, init=torch.from_numpy(init).cuda())
    er, ei = oracle.pagerank(g, 0, 50, 1e-6, init=init)
    assert info["iterations"] == ei["iterations"]
    assert float(np.abs(host(ranks_t, np.float32).astype(np.float64) - er).sum()) <= L1_TOL
    dg.close()
