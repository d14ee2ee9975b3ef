"""Pinning the oracle (CPU, no GPU): the C restatement in oracle/og_oracle.c
must reproduce the reference's outputs bit for bit -- against the committed
golden fixtures (made by tests/golden/make_golden.py from the reference's own
build) and, when oracle/_ref is present, against the reference live."""
import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*_w[01].npz")))
REFERENCE_ROOT = os.environ.get("OGB_REFERENCE_ROOT", "/root/reference")
LAW_ENRON = os.path.join(REFERENCE_ROOT, "01_test_graphs/LAW/LAW-enron/graph.bin")


def test_fixtures_present():
    assert len(FIXTURES) >= 8


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_matches_golden(oracle, path):
    z = dict(np.load(path))
    weighted = path.endswith("_w1.npz")
    s, d = z["src"], z["dst"]
    w = z["w"] if weighted else None
    for sort in range(4):
        es, ed, ew = oracle.sort(s, d, w, 1 if sort in (1, 3) else 0)
        assert np.array_equal(es, z[f"sort{sort}_src"]) and np.array_equal(ed, z[f"sort{sort}_dst"]), sort
        if weighted:
            assert np.array_equal(ew.view(np.uint32), z[f"sort{sort}_w"].view(np.uint32))
    V = int(z["csr_s0_d0_num_vertices"])
    for sort in (0, 1):
        g = oracle.build(s, d, V, sort, w)
        tag = f"csr_s{sort}_d0_"
        for k in ("f_src", "f_dst", "f_outdeg", "f_indeg", "f_idx", "i_src", "i_dst", "i_outdeg", "i_indeg", "i_idx"):
            assert np.array_equal(g[k], z[tag + k]), (sort, k)
        if weighted:
            assert np.array_equal(g["f_w"].view(np.uint32), z[tag + "f_w"].view(np.uint32))
            assert np.array_equal(g["i_w"].view(np.uint32), z[tag + "i_w"].view(np.uint32))
    # dedup path (sort 1 + removeDulpicatesSelfLoopEdges)
    ss, sd, sw = oracle.sort(s, d, w, 1)
    ds, dd, dw = oracle.dedup(ss, sd, sw, truncate_w=weighted)
    g = oracle.build(ds, dd, V, 1, dw)
    for k in ("f_src", "f_dst", "f_outdeg", "f_idx", "i_src", "i_dst", "i_outdeg", "i_idx"):
        assert np.array_equal(g[k], z["csr_s1_d1_" + k]), ("dedup", k)
    if weighted:
        assert np.array_equal(g["f_w"].view(np.uint32), z["csr_s1_d1_f_w"].view(np.uint32))
    # BFS and PageRank on the sort-0 graph
    g = oracle.build(s, d, V, 0, None)
    for mode in (0, 1, 2):
        for i, r in enumerate(z["bfs_roots"]):
            par, dist, st = oracle.bfs(g, int(r), mode)
            assert np.array_equal(dist, z[f"bfs_m{mode}_r{i}_dist"]), (mode, i)
            assert [st["processed_nodes"], st["iteration"]] == list(z[f"bfs_m{mode}_r{i}_stats"])
            if mode == 0:
                assert np.array_equal(par, z[f"bfs_m{mode}_r{i}_par"])
    ranks, st = oracle.pagerank(g, 0, 20, 1e-4)
    assert np.array_equal(ranks.view(np.uint32), z["pr_pull_ranks"].view(np.uint32))
    assert st["iterations"] == int(z["pr_pull_stats"][0])
    assert abs(st["error_total"] - float(z["pr_pull_error"][0])) <= 1e-12


@pytest.mark.parametrize("scale,sort", [(10, 0), (12, 1), (12, 2), (13, 3)])
def test_oracle_matches_reference_live(og, oracle, ref, tmp_path, scale, sort):
    s, d, _ = og.generate_rmat(scale, 16, 7)
    path = str(tmp_path / "g.bin")
    og.write_edge_file(path, s, d)
    rg = ref.build_graph(path, sort=sort)
    ga = og.graph_arrays(rg)
    g = oracle.build(s, d, ga["num_vertices"], sort)
    for k, v in g.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, ga[k]), k
    root = int(np.argmax(ga["f_outdeg"]))
    for mode in (0, 1, 2):
        rp, rd, rs = ref.bfs(rg, root, mode)
        op, od, os_ = oracle.bfs(g, root, mode)
        assert np.array_equal(rd, od)
        assert rs["processed_nodes"] == os_["processed_nodes"] and rs["iteration"] == os_["iteration"]
    rr, rs = ref.pagerank(rg, 0, 30, 1e-6)
    orr, os_ = oracle.pagerank(g, 0, 30, 1e-6)
    assert np.array_equal(rr.view(np.uint32), orr.view(np.uint32))
    assert rs["iterations"] == os_["iterations"]
    ref.graphCSRFree(rg)


@pytest.mark.skipif(not os.path.exists(LAW_ENRON), reason="reference test graph not mounted")
def test_oracle_matches_reference_on_law_enron(og, oracle, ref):
    """The reference's own equivalence-test input (test_open-graph-match.c:59-86:
    LAW-enron, dflag=1 so sort=1)."""
    raw = np.fromfile(LAW_ENRON, dtype=np.uint32).reshape(-1, 2)
    s, d = raw[:, 0].copy(), raw[:, 1].copy()
    rg = ref.build_graph(LAW_ENRON, sort=1, dflag=1)
    ga = og.graph_arrays(rg)
    V = ga["num_vertices"]
    ss, sd, _ = oracle.sort(s, d, None, 1)
    ds, dd, _ = oracle.dedup(ss, sd)
    g = oracle.build(ds, dd, V, 1)
    for k, v in g.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, ga[k]), k
    for root in (int(np.argmax(ga["f_outdeg"])), 0, 12345):
        rp, rd, rs = ref.bfs(rg, root, 2)
        op, od, os_ = oracle.bfs(g, root, 2)
        assert np.array_equal(rd, od)
    rr, rs = ref.pagerank(rg, 0, 100, 1e-6)
    orr, os_ = oracle.pagerank(g, 0, 100, 1e-6)
    assert np.array_equal(rr.view(np.uint32), orr.view(np.uint32)) and rs["iterations"] == os_["iterations"]
    ref.graphCSRFree(rg)


def test_oracle_fp64_close_to_fp32(og, oracle):
    s, d, _ = og.generate_rmat(11, 16, 1)
    V = int(max(s.max(), d.max())) + 1
    g = oracle.build(s, d, V, 0)
    r32, _ = oracle.pagerank(g, 0, 30, 0.0)
    r64 = oracle.pagerank_f64(g, 30)
    assert float(np.abs(r32 - r64).sum()) < 1e-5


def test_oracle_random_roots_match_reference_picker(og, oracle, ref, tmp_path):
    import ctypes as C
    s, d, _ = og.generate_rmat(10, 16, 2)
    path = str(tmp_path / "g.bin")
    og.write_edge_file(path, s, d)
    rg = ref.build_graph(path)
    ga = og.graph_arrays(rg)
    roots = oracle.random_roots(ga["num_vertices"], ga["avg_degree"], ga["f_outdeg"], 20)
    mt = og.mt19937state()
    ref.initializeMersenneState(C.byref(mt), 27491095)
    for r in roots:
        assert ref.d.generateRandomRootGraphCSR(C.byref(mt), rg) == r
    ref.graphCSRFree(rg)


def test_oracle_matches_law_enron_fixture(oracle):
    """The reference's equivalence-test input (committed as
    tests/golden/law_enron.npz by make_law_enron.py from the reference's own
    build): sort 1 + dedup + CSR digests, BFS distances / counts / pull
    parents from the reference's MT19937 roots, PageRank pull ranks
    bit-exact and push ranks within 1e-6 L1."""
    import hashlib

    def digest(a):
        return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)

    z = dict(np.load(os.path.join(GOLDEN, "law_enron.npz")))
    V = int(z["shape"][0])
    ss, sd, _ = oracle.sort(z["src"], z["dst"], None, 1)
    ds, dd, _ = oracle.dedup(ss, sd)
    g = oracle.build(ds, dd, V, 1)
    assert len(ds) == int(z["shape"][1])
    for k in ("f_src", "f_dst", "f_outdeg", "f_indeg", "f_idx", "i_src", "i_dst", "i_outdeg", "i_indeg", "i_idx"):
        assert np.array_equal(digest(g[k]), z["csr_" + k]), k
    for i, r in enumerate(z["roots"]):
        for mode in (0, 1, 2):
            p, dist, st = oracle.bfs(g, int(r), mode)
            assert np.array_equal(digest(dist), z[f"bfs_m{mode}_r{i}_dist"]), (i, mode)
            assert [st["processed_nodes"], st["iteration"]] == list(z[f"bfs_m{mode}_r{i}_stats"]), (i, mode)
            if mode == 0:
                assert np.array_equal(digest(p), z[f"bfs_m{mode}_r{i}_par"]), i
    # pull sums each row sequentially: bit-exact; the reference's push adds
    # with OpenMP atomics in thread order, so it is held to 1e-6 L1
    r, st = oracle.pagerank(g, 0, 100, 1e-4)
    assert st["iterations"] == int(z["pr_pull_stats"][0])
    assert np.array_equal(r.view(np.uint32), z["pr_pull_ranks"].view(np.uint32))
    r, st = oracle.pagerank(g, 1, 100, 1e-4)
    assert st["iterations"] == int(z["pr_push_stats"][0])
    assert float(np.abs(r.astype(np.float64) - z["pr_push_ranks"]).sum()) <= 1e-6


def test_oracle_generator_equals_product_generator(og, oracle):
    """bench.py's reference arm makes its input with the oracle's generator
    (no product library in that process): it must equal the product's
    ogb_generate_rmat bit for bit (both are host code)."""
    for scale, ef, seed, weighted in ((12, 16, 3, True), (10, 8, 0, False), (15, 16, 0, True)):
        a = oracle.generate_rmat(scale, ef, seed, weighted=weighted)
        b = og.generate_rmat(scale, ef, seed, weighted=weighted)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        if weighted:
            assert np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32))


def test_oracle_edge_file_writer_equals_product(og, tmp_path):
    from oracle.oracle import write_edge_file
    s, d, w = og.generate_rmat(10, 8, 1, weighted=True)
    for weighted in (False, True):
        p1, p2 = str(tmp_path / "a"), str(tmp_path / "b")
        write_edge_file(p1, s, d, w if weighted else None)
        og.write_edge_file(p2, s, d, w if weighted else None)
        assert open(p1, "rb").read() == open(p2, "rb").read()


def test_gen_rmat_file_equals_product_file(og, tmp_path):
    """oracle/gen_rmat (what bench.py's reference arm runs to make its input)
    writes the same .wbin / .bin bytes as the product's generator + writer."""
    import subprocess

    from oracle.oracle import HERE
    gen = os.path.join(HERE, "gen_rmat")
    if not os.path.exists(gen):
        subprocess.run(["make", "-s", "-C", HERE, "gen_rmat"], check=True)
    for weighted in (True, False):
        p1, p2 = str(tmp_path / "a"), str(tmp_path / "b")
        subprocess.run([gen, "11", "16", "5", "1" if weighted else "0", p1], check=True)
        s, d, w = og.generate_rmat(11, 16, 5, weighted=weighted)
        og.write_edge_file(p2, s, d, w)
        assert open(p1, "rb").read() == open(p2, "rb").read()


@pytest.mark.parametrize("scale,seed", [(10, 3), (11, 8)])
def test_oracle_dd_and_spmv_match_reference(og, oracle, ref, tmp_path, scale, seed):
    """Data-driven PageRank 6/7/8 (the reference with one kernel thread:
    threaded, its push loses updates and is not reproducible), SPMV pull and
    the sort by rank: bit-exact; SPMV push (omp atomics) within 1e-5."""
    import ctypes as C

    from oracle.oracle import silenced_stdout
    s, d, _ = og.generate_rmat(scale, 16, seed)
    path = str(tmp_path / "g.bin")
    og.write_edge_file(path, s, d)
    rg = ref.build_graph(path)
    ga = og.graph_arrays(rg)
    V = ga["num_vertices"]
    for mode in (6, 7, 8):
        a = ref.arguments(pushpull=mode, iterations=40, epsilon=1e-5)
        a.ker_numThreads = 1
        with silenced_stdout():
            st = ref.pageRankGraphCSR(C.byref(a), rg)
        rr = og.as_numpy(st.contents.pageRanks, V, np.float32)
        rit, rerr = st.contents.iterations, st.contents.error_total
        ref.freePageRankStats(st)
        orr, oi = oracle.pagerank_dd(ga, mode, 40, 1e-5)
        assert np.array_equal(rr.view(np.uint32), orr.view(np.uint32)), mode
        assert rit == oi["iterations"] and rerr == oi["error_total"], mode
    for mode in (0, 1):
        a = ref.arguments(pushpull=mode, iterations=4)
        with silenced_stdout():
            st = ref.SPMVGraphCSR(C.byref(a), rg)
        rx, ry = og.as_numpy(st.contents.vector_input, V, np.float32), og.as_numpy(st.contents.vector_output, V,
                                                                                   np.float32)
        ref.freeSPMVStats(st)
        ox, oy = oracle.spmv(ga, mode, 4)
        assert np.array_equal(rx, ox)
        if mode == 0:
            assert np.array_equal(ry.view(np.uint32), oy.view(np.uint32))
        else:
            assert float((np.abs(ry - oy) / np.maximum(np.abs(oy), 1e-30)).max()) <= 1e-5
    pr, _ = oracle.pagerank(ga, 0, 20, 1e-4)
    lab = np.random.default_rng(seed).permutation(V).astype(np.uint32)
    theirs = lab.copy()
    ref.radixSortEdgesByPageRank(pr.ctypes.data_as(og.f32p), theirs.ctypes.data_as(og.u32p), V)
    assert np.array_equal(theirs, oracle.rank_sort(pr, lab))
    ref.graphCSRFree(rg)


def test_oracle_matches_dd_spmv_fixture(oracle):
    """tests/golden/dd_spmv_rmat10.npz (made by make_golden_dd.py from the
    reference's build): data-driven PageRank 6/7/8, SPMV pull and the sort by
    rank, bit-exact."""
    z = dict(np.load(os.path.join(GOLDEN, "dd_spmv_rmat10.npz")))
    V = int(max(z["src"].max(), z["dst"].max())) + 1
    g = oracle.build(z["src"], z["dst"], V, 0)
    for mode in (6, 7, 8):
        r, st = oracle.pagerank_dd(g, mode, 50, 1e-5)
        assert np.array_equal(r.view(np.uint32), z[f"dd{mode}_ranks"].view(np.uint32)), mode
        assert st["iterations"] == int(z[f"dd{mode}_stats"][0]) and st["error_total"] == float(z[f"dd{mode}_error"][0])
    x, y = oracle.spmv(g, 0, 3)
    assert np.array_equal(x, z["spmv_x"]) and np.array_equal(y.view(np.uint32), z["spmv_y"].view(np.uint32))
    assert np.array_equal(oracle.rank_sort(z["dd6_ranks"], z["sort_labels_in"]), z["sort_labels_out"])


def test_oracle_matches_reference_live_random(og, oracle, ref, tmp_path):
    """Property: on random small edge lists (duplicates, self loops and
    vertices without edges included), every sort type, random roots and all
    three BFS modes, the oracle's CSR arrays, BFS depths and stats and
    PageRank pull ranks equal the reference's own build and search."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=25, deadline=None)
    @given(st.integers(2, 80), st.integers(1, 400), st.sampled_from([0, 1, 2, 3]), st.integers(0, 2**31 - 1))
    def check(V, E, sort, seed):
        rng = np.random.default_rng(seed)
        s = rng.integers(0, V, E).astype(np.uint32)
        d = rng.integers(0, V, E).astype(np.uint32)
        path = str(tmp_path / f"r{seed}.bin")
        og.write_edge_file(path, s, d)
        rg = ref.build_graph(path, sort=sort)
        try:
            ga = og.graph_arrays(rg)
            g = oracle.build(s, d, ga["num_vertices"], sort)
            for k, v in g.items():
                if isinstance(v, np.ndarray):
                    assert np.array_equal(v, ga[k]), k
            for root in {int(rng.integers(0, ga["num_vertices"])), int(np.argmax(ga["f_outdeg"]))}:
                for mode in (0, 1, 2):
                    rp, rd, rs = ref.bfs(rg, root, mode)
                    op, od, os_ = oracle.bfs(g, root, mode)
                    assert np.array_equal(rd, od), (root, mode)
                    assert (rs["processed_nodes"], rs["iteration"]) == (os_["processed_nodes"], os_["iteration"])
            rr, rs = ref.pagerank(rg, 0, 20, 1e-6)
            orr, os_ = oracle.pagerank(g, 0, 20, 1e-6)
            assert np.array_equal(rr.view(np.uint32), orr.view(np.uint32))
            assert rs["iterations"] == os_["iterations"]
        finally:
            ref.graphCSRFree(rg)

    check()
