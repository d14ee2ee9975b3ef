"""GPU parity: PageRank pull and push (pageRank.c:939-1186).

Two bars, both through the C ABI:

1. Pull is deterministic and must be BIT-EXACT against the oracle run in the
   GPU kernel's reduction order (oracle mode 2: rows of <= warp_thr edges
   summed sequentially in CSR order -- the reference's own order -- longer
   rows by the kernel's fixed lane/warp order), ranks and iteration count.
2. Against the reference's sequential order (oracle mode 0/1, itself pinned
   bit-exactly to the reference build), normalized ranks must be within
   L1_TOL = 1e-6 at the same iteration count, on graphs whose rank is not
   concentrated on one hub.  The stop rule (every vertex changes by less
   than epsilon, pageRank.c:1024-1033) is compared at matched iteration
   counts: fp32 rounding flips vertices at the epsilon boundary, so the
   iteration at which it fires may differ by a few.

The "star" graph (64 vertices, one hub with ~20k in-edges holding half of the
rank) is the documented exception to bar 2: there summation order alone
moves the L1 by ~5e-5 (the same amount a CPU emulation of the GPU order
shows), so it is held to bar 1 only, and to STAR_TOL (STAR_TOL_PUSH for the
atomic push) against the reference order."""
import ctypes as C

import numpy as np
import pytest

from test_build_gpu import dev, host

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6
STAR_TOL = 1e-4        # star, pull: fixed order differs from the sequential one
STAR_TOL_PUSH = 1e-3   # star, push: float atomics in arbitrary order on the hub

CASES = [
    ("rmat", dict(scale=12, ef=16, seed=1)),
    ("rmat", dict(scale=16, ef=16, seed=0)),
    ("uniform", dict(n=40_000, m=200_000, seed=3)),
    ("grid", dict(side=80, p=0.01, seed=2)),
    ("star", dict(n=20_000, seed=4)),
]
IDS = [f"{k}-{i}" for i, (k, _) in enumerate(CASES)]


def bins(lib):
    w, c, t, k = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    lib.ogb_pagerank_get_bins(C.byref(w), C.byref(c), C.byref(t), C.byref(k))
    return w.value, c.value, t.value, k.value


@pytest.fixture
def setup(torch_cuda, lib, oracle, graphs):
    def make(kind, kw):
        s, d, _, V = graphs(kind, **kw)
        g = oracle.build(s, d, V, 0)
        dg = lib.device_graph()
        dg.build(dev(torch_cuda, s), dev(torch_cuda, d), V, 0)
        return g, dg, V
    return make


@pytest.mark.parametrize("kind,kw", CASES, ids=IDS)
def test_pull_bitexact_vs_gpu_order_oracle(torch_cuda, lib, oracle, setup, kind, kw):
    g, dg, V = setup(kind, kw)
    oracle.set_gpu_order(*bins(lib))
    ranks_t = torch_cuda.empty(V, dtype=torch_cuda.float32, device="cuda")
    for iters, eps in ((20, 0.0), (100, 1e-4), (100, 1e-6)):
        info = dg.pagerank(ranks_t, mode=0, max_iterations=iters, epsilon=eps)
        er, ei = oracle.pagerank(g, 2, iters, eps)
        assert np.array_equal(host(ranks_t, np.float32).view(np.uint32), er.view(np.uint32)), (iters, eps)
        assert info["iterations"] == ei["iterations"]
        errs, act = dg.pagerank_history()
        assert np.array_equal(act, ei["active_hist"])
        assert np.allclose(errs, ei["err_hist"], rtol=1e-12, atol=0)
    dg.close()


@pytest.mark.parametrize("kind,kw", CASES, ids=IDS)
@pytest.mark.parametrize("mode", [0, 1])
def test_l1_vs_reference_order(torch_cuda, lib, oracle, setup, kind, kw, mode):
    g, dg, V = setup(kind, kw)
    tol = (STAR_TOL_PUSH if mode == 1 else STAR_TOL) if kind == "star" else L1_TOL
    ranks_t = torch_cuda.empty(V, dtype=torch_cuda.float32, device="cuda")
    # fixed iteration count
    dg.pagerank(ranks_t, mode=mode, max_iterations=20, epsilon=0.0)
    er, _ = oracle.pagerank(g, mode, 20, 0.0)
    l1 = float(np.abs(host(ranks_t, np.float32).astype(np.float64) - er).sum())
    assert l1 <= tol, l1
    # the reference's stop rule: compare at the iteration count our run used
    info = dg.pagerank(ranks_t, mode=mode, max_iterations=100, epsilon=1e-4)
    er, ei_stop = oracle.pagerank(g, mode, 100, 1e-4)
    er_m, _ = oracle.pagerank(g, mode, info["executed"], 0.0)
    l1 = float(np.abs(host(ranks_t, np.float32).astype(np.float64) - er_m).sum())
    assert l1 <= tol, (l1, info["executed"])
    print(f"{kind} mode {mode}: stop-rule iterations gpu {info['iterations']} vs reference order "
          f"{ei_stop['iterations']}; L1 at matched count {l1:.2e}")
    dg.close()


def test_fp64_error_stated(torch_cuda, lib, oracle, setup):
    g, dg, V = setup("rmat", dict(scale=14, ef=16, seed=2))
    ranks_t = torch_cuda.empty(V, dtype=torch_cuda.float32, device="cuda")
    dg.pagerank(ranks_t, mode=0, max_iterations=30, epsilon=0.0)
    r64 = oracle.pagerank_f64(g, 30)
    r32, _ = oracle.pagerank(g, 0, 30, 0.0)
    gpu = host(ranks_t, np.float32).astype(np.float64)
    l1_gpu, l1_ref = float(np.abs(gpu - r64).sum()), float(np.abs(r32 - r64).sum())
    print(f"L1 vs FP64 after 30 iterations: GPU {l1_gpu:.3e}, reference fp32 order {l1_ref:.3e}")
    assert l1_gpu < 1e-5 and l1_gpu < 4 * l1_ref + 1e-7
    dg.close()


def test_init_vector(torch_cuda, lib, oracle, setup):
    g, dg, V = setup("rmat", dict(scale=12, ef=16, seed=1))
    oracle.set_gpu_order(*bins(lib))
    init = np.random.default_rng(0).uniform(0.1, 2.0, V).astype(np.float32)
    ranks_t = torch_cuda.empty(V, dtype=torch_cuda.float32, device="cuda")
    info = dg.pagerank(ranks_t, mode=0, max_iterations=50, epsilon=1e-6, init=torch_cuda.from_numpy(init).cuda())
    er, ei = oracle.pagerank(g, 2, 50, 1e-6, init=init)
    assert info["iterations"] == ei["iterations"]
    assert np.array_equal(host(ranks_t, np.float32).view(np.uint32), er.view(np.uint32))
    dg.close()


def test_bins_are_settable(torch_cuda, lib, oracle, setup):
    """Other thresholds change the order of the heavy rows only; the oracle
    follows them bit for bit."""
    g, dg, V = setup("rmat", dict(scale=14, ef=16, seed=5))
    saved = bins(lib)
    try:
        for wt, ct in ((8, 256), (64, 100000), (0, 0)):
            lib.ogb_pagerank_set_bins(wt, ct)
            oracle.set_gpu_order(*bins(lib))
            ranks_t = torch_cuda.empty(V, dtype=torch_cuda.float32, device="cuda")
            dg.pagerank(ranks_t, mode=0, max_iterations=10, epsilon=0.0)
            er, _ = oracle.pagerank(g, 2, 10, 0.0)
            assert np.array_equal(host(ranks_t, np.float32).view(np.uint32), er.view(np.uint32)), (wt, ct)
    finally:
        lib.ogb_pagerank_set_bins(saved[0], saved[1])
        dg.close()
