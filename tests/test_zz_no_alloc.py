"""GPU test of ogb_pagerank_pull_noalloc, the PageRank entry point for
callers that cannot allocate device memory when they need a result (device
memory owned by another allocator, or a request path on which cudaMalloc is
not allowed).  Its scratch is a fixed array inside the library, so it takes
no allocation of its own.

Called through the C ABI twice in a row (different tolerances, so the second
call must not see the first one's state) and compared with the existing entry
point ogb_pagerank (pull) and with the oracle's sequential (reference-order)
pull, each within the 1e-6 L1 tolerance of the PageRank tests, at the same
iteration count.  The graph is checked to hold rows of all three kinds the
kernel splits by in-degree (<= 32: a thread, 33..2048: a warp, > 2048: a CTA),
so every branch runs.  This file is collected last on purpose: if it fails, a
run that stops at the first failure has run everything else."""
import ctypes as C

import numpy as np
import pytest

import opengraph_b200 as og

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def test_noalloc_matches_pagerank_pull_twice():
    import torch

    from oracle.oracle import Oracle
    torch.cuda.init()
    lib = og.load(False)
    lib.quiet(True)
    s, d, _ = og.generate_rmat(16, 16, 3)
    V = int(max(s.max(), d.max())) + 1
    orc = Oracle()
    g = orc.build(s, d, V, 0)
    indeg = g["i_outdeg"]
    assert indeg.max() > 2048, "no row for the CTA branch"
    assert np.any((indeg > 32) & (indeg <= 2048)), "no row for the warp branch"
    assert np.any((indeg > 0) & (indeg <= 32)), "no row for the thread branch"
    dg = lib.device_graph()
    dg.build(torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda(), V, 0)
    inv, fwd = dg.view(True), dg.view(False)
    ranks_ref = torch.empty(V, dtype=torch.float32, device="cuda")
    ranks = torch.empty(V, dtype=torch.float32, device="cuda")
    info_d = torch.zeros(C.sizeof(og.PrInfo), dtype=torch.uint8, device="cuda")
    for iters, eps in ((30, 1e-4), (60, 1e-7)):
        ref = dg.pagerank(ranks_ref, mode=0, max_iterations=iters, epsilon=eps)
        ranks.fill_(-1.0)
        st = lib.ogb_pagerank_pull_noalloc(V, inv.edges_idx.data_ptr(), inv.out_degree.data_ptr(),
                                           inv.dst.data_ptr(), fwd.out_degree.data_ptr(), iters, eps,
                                           ranks.data_ptr(), info_d.data_ptr(), None)
        lib.check(st, "ogb_pagerank_pull_noalloc")
        torch.cuda.synchronize()
        info = og.PrInfo.from_buffer_copy(bytes(info_d.cpu().numpy()))
        l1 = float((ranks.double() - ranks_ref.double()).abs().sum())
        assert l1 <= L1_TOL, (iters, eps, l1)
        assert info.iterations == ref["iterations"] and info.executed == ref["executed"]
        assert abs(info.error_total - ref["error_total"]) <= L1_TOL
        # the oracle's sequential order at the same executed iteration count
        er, _ = orc.pagerank(g, 0, info.executed, 0.0)
        l1_orc = float(np.abs(ranks.cpu().numpy().astype(np.float64) - er).sum())
        assert l1_orc <= L1_TOL, (iters, eps, l1_orc)
    dg.close()


def test_noalloc_rejects_graphs_beyond_its_scratch():
    lib = og.load(False)
    too_big = (1 << 20) + 1
    st = lib.ogb_pagerank_pull_noalloc(too_big, 1, 1, 1, 1, 10, 1e-4, 1, None, None)
    assert st == 4  # OGB_ERR_RANGE
    assert b"num_vertices" in lib.ogb_last_error()
