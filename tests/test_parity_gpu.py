"""GPU parity on the reference's own test input, on the committed golden
fixtures, and at the benchmarked size.

* LAW-enron (tests/golden/law_enron.npz, made by make_law_enron.py from the
  reference's CPU build): the reference's equivalence-test configuration
  (test_open-graph-match.c:59-86 -- dflag=1, sort=1, roots from MT19937 seed
  27491095, 100 iterations, epsilon 1e-4) through the drop-in C API:
  graphCSRPreProcessingStep, breadthFirstSearchGraphCSR (pushpull 0/1/2) and
  pageRankGraphCSR (pull, push).
* Every tests/golden/<graph>_w{0,1}.npz through the drop-in C API: the four
  SORT_TYPEs, the CSR with and without dedup, BFS in three modes from the
  fixture's roots, PageRank pull.
* RMAT scale 22 (V = 4,194,304, E = 67,108,864, float32 weights: the
  benchmark's graph, seed 0) against the oracle: the CSR of both directions
  for sort 0 (drop-in build) and sort 1 (device API), bit-exact; DO-BFS from
  the benchmark's first roots (depths, iteration and processed counts, TD/BU
  step sequence, valid parents); PageRank pull and push to epsilon 1e-6
  (max 100 iterations) within 1e-6 L1 of the reference order at the same
  iteration count, with the error against FP64 printed.

Bars: CSR arrays, sort outputs, distances and counts bit-exact; parents valid
(bottom-up-only parents equal); ranks within L1_TOL = 1e-6."""
import ctypes as C
import glob
import hashlib
import os

import numpy as np
import pytest

from test_build_gpu import dev, host

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LAW = os.path.join(GOLDEN, "law_enron.npz")
FIXTURES = sorted(f for f in glob.glob(os.path.join(GOLDEN, "*_w[01].npz")))
CSR_KEYS = ("f_src", "f_dst", "f_outdeg", "f_indeg", "f_idx", "i_src", "i_dst", "i_outdeg", "i_indeg", "i_idx")


def digest(a):
    a = np.ascontiguousarray(a)
    return np.frombuffer(hashlib.sha256(a.astype(a.dtype.newbyteorder("<")).tobytes()).digest(), np.uint8)


def dropin_graph(og, lib, path, **kw):
    a = og.default_arguments(fnameb=path, **kw)
    lib.initializeMersenneState(C.byref(a.mt19937var), 27491095)
    return lib.graphCSRPreProcessingStep(C.byref(a))


def dropin_bfs(og, lib, g, root, pushpull):
    a = og.default_arguments(source=int(root), pushpull=pushpull)
    st = lib.breadthFirstSearchGraphCSR(C.byref(a), g)
    s = st.contents
    V = s.num_vertices
    out = (og.as_numpy(s.parents, V, np.int32), og.as_numpy(s.distances, V, np.uint32),
           {"processed_nodes": s.processed_nodes, "iteration": s.iteration})
    lib.freeBFSStats(st)
    return out


def dropin_pagerank(og, lib, g, pushpull, iterations, epsilon):
    a = og.default_arguments(pushpull=pushpull, iterations=iterations, epsilon=epsilon)
    st = lib.pageRankGraphCSR(C.byref(a), g)
    s = st.contents
    out = (og.as_numpy(s.pageRanks, s.num_vertices, np.float32),
           {"iterations": s.iterations, "error_total": s.error_total})
    lib.freePageRankStats(st)
    return out


def check_parents_full(g, root, par, dist):
    """Every reached vertex's parent is an in-neighbour one level up (all
    vertices, vectorised over the inverse CSR); the root is its own parent;
    unreached vertices keep distance 0 and the -out_degree / -1 sentinel."""
    outdeg = g["f_outdeg"]
    reached = par >= 0
    assert par[root] == root and dist[root] == 0
    sentinel = np.where(outdeg > 0, -outdeg.astype(np.int64), -1)
    assert np.array_equal(par[~reached].astype(np.int64), sentinel[~reached])
    assert np.all(dist[~reached] == 0)
    v = np.nonzero(reached)[0]
    v = v[v != root]
    p = par[v].astype(np.int64)
    assert np.all((p >= 0) & (p < g["num_vertices"]))
    assert np.all(dist[p].astype(np.int64) + 1 == dist[v])
    keys = (g["i_src"].astype(np.uint64) << np.uint64(32)) | g["i_dst"].astype(np.uint64)
    if not np.all(keys[1:] >= keys[:-1]):
        keys = np.sort(keys)
    want = (v.astype(np.uint64) << np.uint64(32)) | p.astype(np.uint64)
    pos = np.minimum(np.searchsorted(keys, want), len(keys) - 1)
    assert np.all(keys[pos] == want), "a parent is not an in-neighbour"


# --------------------------------------------------------------- LAW-enron --

@pytest.fixture(scope="module")
def law(tmp_path_factory):
    z = dict(np.load(LAW))
    path = str(tmp_path_factory.mktemp("law") / "law_enron.bin")
    rec = np.stack([z["src"], z["dst"]], axis=1).astype("<u4")
    rec.tofile(path)
    return z, path


def test_law_enron_dropin_csr_bfs(og, lib, oracle, law):
    z, path = law
    g = dropin_graph(og, lib, path, sort=1, dflag=1)
    ga = og.graph_arrays(g)
    assert [ga["num_vertices"], ga["num_edges"], ga["avg_degree"]] == list(z["shape"])
    for k in CSR_KEYS:
        assert np.array_equal(digest(ga[k]), z["csr_" + k]), k
    for i, r in enumerate(z["roots"]):
        for mode in (0, 1, 2):
            par, dist, st = dropin_bfs(og, lib, g, r, mode)
            assert np.array_equal(digest(dist), z[f"bfs_m{mode}_r{i}_dist"]), (i, mode)
            assert [st["processed_nodes"], st["iteration"]] == list(z[f"bfs_m{mode}_r{i}_stats"]), (i, mode)
            if mode == 0:
                assert np.array_equal(digest(par), z[f"bfs_m{mode}_r{i}_par"]), i
            check_parents_full(ga, int(r), par, dist)
    lib.graphCSRFree(g)


@pytest.mark.parametrize("pushpull,tag", [(0, "pull"), (1, "push")])
def test_law_enron_dropin_pagerank(og, lib, oracle, law, pushpull, tag):
    z, path = law
    g = dropin_graph(og, lib, path, sort=1, dflag=1)
    ga = og.graph_arrays(g)
    pr, st = dropin_pagerank(og, lib, g, pushpull, 100, 1e-4)
    ref_it = int(z[f"pr_{tag}_stats"][0])
    if st["iterations"] == ref_it:
        want = z[f"pr_{tag}_ranks"].astype(np.float64)
    else:  # the stop rule fired a few iterations apart in fp32: match the count
        want, _ = oracle.pagerank(ga, pushpull, st["iterations"] + 1, 0.0)
    l1 = float(np.abs(pr.astype(np.float64) - want).sum())
    print(f"LAW-enron {tag}: iterations {st['iterations']} (reference {ref_it}), L1 {l1:.2e}")
    assert abs(st["iterations"] - ref_it) <= 3
    assert l1 <= L1_TOL, l1
    lib.graphCSRFree(g)


# ---------------------------------------------------------- golden fixtures --

@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_golden_fixture_through_dropin(og, lib, libw, tmp_path, path):
    z = dict(np.load(path))
    weighted = path.endswith("_w1.npz")
    L = libw if weighted else lib
    s, d = z["src"], z["dst"]
    w = z["w"] if weighted else None
    f = str(tmp_path / ("g.wbin" if weighted else "g.bin"))
    og.write_edge_file(f, s, d, w)
    wflag = 1 if weighted else 0
    # sortRunAlgorithms, SORT_TYPE 0..3 (GPU sort)
    for sort in range(4):
        el = L.sortRunAlgorithms(L.readEdgeListsbin(f.encode(), 0, 0, wflag), sort)
        ea = og.edge_list_arrays(el)
        assert np.array_equal(ea["src"], z[f"sort{sort}_src"]) and np.array_equal(ea["dst"], z[f"sort{sort}_dst"])
        if weighted:
            assert np.array_equal(ea["w"].view(np.uint32), z[f"sort{sort}_w"].view(np.uint32))
        L.freeEdgeList(el)
    # graphCSRPreProcessingStep with and without dedup
    for sort, dflag in ((0, 0), (1, 0), (1, 1)):
        g = dropin_graph(og, L, f, sort=sort, dflag=dflag, weighted=wflag)
        ga = og.graph_arrays(g)
        tag = f"csr_s{sort}_d{dflag}_"
        for k, v in ga.items():
            want = z[tag + k]
            if isinstance(v, np.ndarray):
                assert np.array_equal(v.view(np.uint32), want.view(np.uint32)), (tag, k)
            else:
                assert v == want, (tag, k)
        if sort == 0 and dflag == 0:
            for i, r in enumerate(z["bfs_roots"]):
                for mode in (0, 1, 2):
                    par, dist, st = dropin_bfs(og, L, g, r, mode)
                    assert np.array_equal(dist, z[f"bfs_m{mode}_r{i}_dist"]), (i, mode)
                    assert [st["processed_nodes"], st["iteration"]] == list(z[f"bfs_m{mode}_r{i}_stats"])
                    if mode == 0:
                        assert np.array_equal(par, z[f"bfs_m{mode}_r{i}_par"])
                    check_parents_full(ga, int(r), par, dist)
            pr, st = dropin_pagerank(og, L, g, 0, 20, 1e-4)
            assert st["iterations"] == int(z["pr_pull_stats"][0])
            assert float(np.abs(pr.astype(np.float64) - z["pr_pull_ranks"]).sum()) <= L1_TOL
            assert abs(st["error_total"] - float(z["pr_pull_error"][0])) <= L1_TOL
        L.graphCSRFree(g)


# ------------------------------------------------ RMAT-22, the bench graph --

SCALE, EF, SEED = 22, 16, 0


@pytest.fixture(scope="module")
def rmat22(oracle):
    s, d, w = oracle.generate_rmat(SCALE, EF, SEED, weighted=True)
    V = 1 << SCALE
    g = oracle.build(s, d, V, 0, w)
    return s, d, w, V, g


@pytest.mark.slow
def test_scale22_csr_sort0_dropin(og, libw, rmat22, tmp_path):
    """graphCSRPreProcessingStep on the bench's .wbin (sort 0): all twelve CSR
    arrays plus both weight arrays equal the oracle's, and DO-BFS through
    breadthFirstSearchGraphCSR (packed result, host expansion) from two
    bench roots equals the oracle."""
    from bench import rank_roots
    from oracle.oracle import Oracle
    s, d, w, V, g = rmat22
    f = str(tmp_path / "rmat22.wbin")
    og.write_edge_file(f, s, d, w)
    gh = dropin_graph(og, libw, f, sort=0, weighted=1)
    ga = og.graph_arrays(gh)
    assert ga["num_vertices"] == V and ga["num_edges"] == len(s)
    for k in CSR_KEYS + ("f_w", "i_w"):
        assert np.array_equal(ga[k].view(np.uint32), g[k].view(np.uint32)), k
    orc = Oracle()
    for r in rank_roots(g["f_outdeg"], 0)[:2]:
        par, dist, st = dropin_bfs(og, libw, gh, r, 2)
        _, edist, est = orc.bfs(g, r, 2)
        assert np.array_equal(dist, edist), r
        assert st["processed_nodes"] == est["processed_nodes"] and st["iteration"] == est["iteration"]
        check_parents_full(g, r, par, dist)
    libw.graphCSRFree(gh)
    os.remove(f)


@pytest.mark.slow
def test_scale22_csr_sort1_device(torch_cuda, libw, oracle, rmat22):
    """ogb_graph_build with sort 1 ((src, dst) order): both directions
    bit-exact against the oracle."""
    torch = torch_cuda
    s, d, w, V, _ = rmat22
    e = oracle.build(s, d, V, 1, w)
    dg = libw.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 1, weight=dev(torch, w))
    for tag, inv in (("f", False), ("i", True)):
        v = dg.view(inv)
        for name, arr in (("src", v.src), ("dst", v.dst), ("outdeg", v.out_degree), ("indeg", v.in_degree),
                          ("idx", v.edges_idx)):
            assert np.array_equal(host(arr), e[f"{tag}_{name}"]), (tag, name)
        assert np.array_equal(host(v.weight, np.float32).view(np.uint32), e[f"{tag}_w"].view(np.uint32)), tag
    dg.close()


@pytest.fixture(scope="module")
def dev22(torch_cuda, libw, rmat22):
    torch = torch_cuda
    s, d, w, V, _ = rmat22
    dg = libw.device_graph()
    dg.build(dev(torch, s), dev(torch, d), V, 0, weight=dev(torch, w))
    yield dg
    dg.close()


@pytest.mark.slow
def test_scale22_dobfs_bench_roots(torch_cuda, oracle, rmat22, dev22):
    """DO-BFS (mode 2) from the bench's first four roots and the hub:
    depths, BFSStats counts and the TD/BU step sequence equal the oracle's;
    parents valid.  The hub also runs pull-only (parents equal) and
    push-only."""
    from bench import rank_roots
    torch = torch_cuda
    _, _, _, V, g = rmat22
    par_t = torch.empty(V, dtype=torch.int32, device="cuda")
    dist_t = torch.empty(V, dtype=torch.int32, device="cuda")
    hub = int(np.argmax(g["f_outdeg"]))
    runs = [(r, 2) for r in rank_roots(g["f_outdeg"], 0)[:4]] + [(hub, 2), (hub, 0), (hub, 1)]
    for root, mode in runs:
        info = dev22.bfs(root, par_t, dist_t, mode=mode)
        par, dist = host(par_t, np.int32), host(dist_t)
        epar, edist, est = oracle.bfs(g, root, mode)
        assert np.array_equal(dist, edist), (root, mode)
        for k in ("iteration", "processed_nodes", "td_steps", "bu_steps", "reached", "reached_out_edges"):
            assert info[k] == est[k], (root, mode, k)
        assert [t["direction"] for t in dev22.bfs_trace()] == list(est["dirs"]), (root, mode)
        check_parents_full(g, root, par, dist)
        if mode == 0:
            assert np.array_equal(par, epar)


@pytest.mark.slow
@pytest.mark.parametrize("mode", [0, 1])
def test_scale22_pagerank_to_1e6(torch_cuda, oracle, rmat22, dev22, mode):
    """PageRank (pull 0 / push 1) with the reference's stop rule at epsilon
    1e-6, at most 100 iterations: normalized ranks within 1e-6 L1 of the
    oracle's sequential (reference) order at the same executed iteration
    count; the L1 against the FP64 restatement is printed."""
    torch = torch_cuda
    _, _, _, V, g = rmat22
    ranks_t = torch.empty(V, dtype=torch.float32, device="cuda")
    info = dev22.pagerank(ranks_t, mode=mode, max_iterations=100, epsilon=1e-6)
    got = host(ranks_t, np.float32).astype(np.float64)
    er, ei = oracle.pagerank(g, mode, info["executed"], 0.0)
    l1 = float(np.abs(got - er).sum())
    msg = f"RMAT-22 PR mode {mode}: executed {info['executed']}, L1 vs reference order {l1:.3e}"
    if mode == 0:
        r64 = oracle.pagerank_f64(g, info["executed"])
        msg += (f", vs FP64 GPU {float(np.abs(got - r64).sum()):.3e} "
                f"/ reference fp32 order {float(np.abs(er - r64).sum()):.3e}")
    print(msg)
    assert l1 <= L1_TOL, msg
