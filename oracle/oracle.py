"""Oracle of the OpenGraph CSR hot path -- TEST INFRASTRUCTURE ONLY.

Two checkers, both CPU:

* ``Oracle``: the project's C restatement (``og_oracle.c`` -> ``liboracle.so``),
  sequential and deterministic, every function citing the reference lines it
  restates;
* ``Reference``: the reference's own OpenMP code compiled from its sources by
  ``oracle/Makefile`` into ``oracle/_ref/libogref{,_w}.so`` (git-ignored build
  output that travels with the tree).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker or the timed CPU baseline; the product
(``opengraph_b200``) never imports it.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# the reference tree (read only where it is mounted; override with OGB_REFERENCE_ROOT)
REFERENCE_ROOT = os.environ.get("OGB_REFERENCE_ROOT", "/root/reference")
REFERENCE_SRC = os.path.join(REFERENCE_ROOT, "00_graph_bench")

u32 = C.c_uint32
vp = C.c_void_p


def build(ref: bool = True) -> None:
    """make the restatement (and, when the reference sources exist, _ref)."""
    targets = ["oracle"]
    if ref and os.path.isdir(REFERENCE_SRC):
        targets.append("ref")
        # the reference's driver, as shipped and linked to the product library
        if os.path.exists(os.path.join(HERE, "..", "opengraph_b200", "libogb200.so")):
            targets.append("driver")
    subprocess.run(["make", "-s", "-C", HERE, "-j8", f"REF={REFERENCE_SRC}", *targets], check=True)


def _p(a):
    return None if a is None else a.ctypes.data


class Oracle:
    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        d = C.CDLL(path)
        self.d = d
        d.orc_sort.argtypes = [u32, vp, vp, vp, C.c_int, vp, vp, vp]
        d.orc_csr_map.argtypes = [u32, u32, vp, vp, vp]
        d.orc_csr_map.restype = C.c_int
        d.orc_build.argtypes = [u32, u32, vp, vp, vp, C.c_int] + [vp] * 12
        d.orc_build.restype = C.c_int
        d.orc_dedup.argtypes = [u32, vp, vp, vp, vp, vp, vp, C.c_int]
        d.orc_dedup.restype = u32
        d.orc_bfs.argtypes = [u32, u32, vp, vp, vp, vp, vp, vp, u32, C.c_int, C.c_int, vp, vp, vp, vp, u32]
        d.orc_bfs.restype = C.c_int
        d.orc_pagerank.argtypes = [u32, vp, vp, vp, vp, vp, vp, C.c_int, u32, C.c_double, vp, vp, vp, vp, vp, vp]
        d.orc_pagerank.restype = u32
        d.orc_pagerank_f64.argtypes = [u32, vp, vp, vp, vp, u32, vp, vp]
        d.orc_random_roots.argtypes = [u32, u32, u32, vp, u32, vp]
        d.orc_set_gpu_order.argtypes = [u32, u32, u32, u32]
        d.orc_generate_rmat.argtypes = [u32, u32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_int, vp, vp,
                                        vp]
        d.orc_generate_rmat.restype = C.c_int
        d.orc_pagerank_dd.argtypes = [u32, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, u32, C.c_double, vp, vp, vp, vp]
        d.orc_pagerank_dd.restype = u32
        d.orc_spmv.argtypes = [u32, vp, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, u32, vp, vp]
        d.orc_rank_sort.argtypes = [u32, vp, vp]
        d.orc_pull_range_step.argtypes = [u32, vp, vp, vp, vp, u32, u32, vp, vp, vp, C.c_double, C.c_int, vp, vp]
        d.orc_bfs_range_init.argtypes = [u32, vp, u32, u32, u32, vp, vp, vp, vp, vp]
        d.orc_bfs_range_expand.argtypes = [u32, vp, vp, vp, vp, vp, vp, u32, u32, C.c_int, u32, vp, vp, vp, vp, vp,
                                           vp, vp]
        d.orc_bfs_range_settle.argtypes = [u32, vp, u32, u32, C.c_int, u32, vp, vp, vp, vp, vp, vp]

    def pull_range_step(self, g: dict, lo: int, hi: int, contrib, pr, contrib_next, epsilon: float,
                        gpu_order: bool = True):
        """One pull iteration over [lo, hi) (numpy float32 arrays of V, in
        place); returns the range's (error, active)."""
        err, act = C.c_double(0.0), u32(0)
        self.d.orc_pull_range_step(g["num_vertices"], _p(g["f_outdeg"]), _p(g["i_outdeg"]), _p(g["i_idx"]),
                                   _p(g["i_dst"]), lo, hi, _p(contrib), _p(pr), _p(contrib_next), epsilon,
                                   1 if gpu_order else 0, C.byref(err), C.byref(act))
        return err.value, act.value

    def bfs_range_init(self, g: dict, lo: int, hi: int, root: int, parents, dist, frontier, visited, cand) -> int:
        """One rank's initialisation of the partitioned DO-BFS (numpy arrays
        of V, in place); returns the root's out-degree (the first mf)."""
        self.d.orc_bfs_range_init(g["num_vertices"], _p(g["f_outdeg"]), lo, hi, root, _p(parents), _p(dist),
                                  _p(frontier), _p(visited), _p(cand))
        return int(g["f_outdeg"][root])

    def bfs_range_expand(self, g: dict, lo: int, hi: int, direction: int, depth: int, frontier, visited, nxt,
                         cand, parents, dist, counts) -> None:
        self.d.orc_bfs_range_expand(g["num_vertices"], _p(g["f_outdeg"]), _p(g["f_idx"]), _p(g["f_dst"]),
                                    _p(g["i_outdeg"]), _p(g["i_idx"]), _p(g["i_dst"]), lo, hi, direction, depth,
                                    _p(frontier), _p(visited), _p(nxt), _p(cand), _p(parents), _p(dist), _p(counts))

    def bfs_range_settle(self, g: dict, lo: int, hi: int, direction: int, depth: int, cand, nxt, visited,
                         parents, dist, counts) -> None:
        self.d.orc_bfs_range_settle(g["num_vertices"], _p(g["f_outdeg"]), lo, hi, direction, depth, _p(cand),
                                    _p(nxt), _p(visited), _p(parents), _p(dist), _p(counts))

    @staticmethod
    def partition_edges(src, dst, w, bounds):
        """Stable split of an edge shard by vertex owner (owner r holds
        [bounds[r], bounds[r+1])): per owner in rank order, the edges it owns
        by source, then those it owns by destination only, each in shard
        order.  Returns (src, dst, w or None, counts per owner).  The
        graph-build exchange of a 1-D partition; the reference builds one
        graph in one process (graphCSR.c:107-248)."""
        b = np.asarray(bounds, np.int64)
        s64, d64 = np.asarray(src, np.int64), np.asarray(dst, np.int64)
        if len(s64) and max(int(s64.max()), int(d64.max())) >= b[-1]:
            raise ValueError("partition: a vertex id is past the last range")
        os_ = np.searchsorted(b, s64, side="right") - 1
        od = np.searchsorted(b, d64, side="right") - 1
        idx, counts = [], []
        for r in range(len(b) - 1):
            a = np.nonzero(os_ == r)[0]
            c = np.nonzero((od == r) & (os_ != r))[0]
            idx.append(a)
            idx.append(c)
            counts.append(len(a) + len(c))
        k = np.concatenate(idx) if idx else np.zeros(0, np.int64)
        return (np.asarray(src)[k], np.asarray(dst)[k], (np.asarray(w)[k] if w is not None else None), counts)

    def pagerank_dd(self, g: dict, mode: int, max_iters: int = 100, epsilon: float = 1e-4, gpu_order: bool = False):
        """Data-driven PageRank (6 pull, 7 push, 8 pull-push), sequential;
        gpu_order sums long in-rows as the GPU kernels do (mode 6)."""
        V = g["num_vertices"]
        ranks = np.empty(V, np.float32)
        it, err = u32(), C.c_double()
        ah = np.zeros(max(max_iters, 1), np.uint32)
        n = self.d.orc_pagerank_dd(V, _p(g["f_outdeg"]), _p(g["f_idx"]), _p(g["f_dst"]), _p(g["i_outdeg"]),
                                   _p(g["i_idx"]), _p(g["i_dst"]), mode, 1 if gpu_order else 0, max_iters, epsilon,
                                   _p(ranks), C.byref(it), C.byref(err), _p(ah))
        return ranks, {"iterations": it.value, "error_total": err.value, "executed": n, "active_hist": ah[:n]}

    def spmv(self, g: dict, mode: int = 0, iters: int = 20, weighted: bool = False, gpu_order: bool = False):
        """SPMV pull (0) / push (1), sequential; weights from the graph dict
        (i_w for pull, f_w for push) when weighted, else 0.0001 each."""
        V = g["num_vertices"]
        x, y = np.empty(V, np.float32), np.empty(V, np.float32)
        w = (g["i_w"] if mode == 0 else g["f_w"]) if weighted else None
        self.d.orc_spmv(V, _p(g["f_outdeg"]), _p(g["f_idx"]), _p(g["f_dst"]), _p(g["i_outdeg"]), _p(g["i_idx"]),
                        _p(g["i_dst"]), _p(w), mode, 1 if gpu_order else 0, iters, _p(x), _p(y))
        return x, y

    def rank_sort(self, ranks, labels):
        """radixSortEdgesByPageRank: the labels sorted by fixed-point rank."""
        r = np.ascontiguousarray(ranks, np.float32)
        out = np.ascontiguousarray(labels, np.uint32).copy()
        self.d.orc_rank_sort(len(out), _p(r), _p(out))
        return out

    def generate_rmat(self, scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19, permute=True,
                      weighted=False):
        """The benchmark's seeded RMAT edge list, made without the product
        library (equal to opengraph_b200.generate_rmat bit for bit)."""
        E = (1 << scale) * edge_factor
        src, dst = np.empty(E, np.uint32), np.empty(E, np.uint32)
        w = np.empty(E, np.float32) if weighted else None
        if self.d.orc_generate_rmat(scale, edge_factor, seed, a, b, c, 1 if permute else 0, _p(src), _p(dst), _p(w)):
            raise ValueError("oracle generate_rmat: bad sizes")
        return src, dst, w

    def set_gpu_order(self, warp_thr: int = 32, cta_thr: int = 2048, cta_threads: int = 256,
                      chunk: int = 8192) -> None:
        """Reduction order that pagerank(mode=2) emulates (the GPU pull kernel's work split)."""
        self.d.orc_set_gpu_order(warp_thr, cta_thr, cta_threads, chunk)

    def sort(self, src, dst, w=None, mode: int = 0):
        E = len(src)
        os_, od = np.empty(E, np.uint32), np.empty(E, np.uint32)
        ow = np.empty(E, np.float32) if w is not None else None
        self.d.orc_sort(E, _p(src), _p(dst), _p(w), mode, _p(os_), _p(od), _p(ow))
        return os_, od, ow

    def build(self, src, dst, V: int, sort_type: int = 0, w=None) -> dict:
        E = len(src)
        r = {k: np.empty(E, np.uint32) for k in ("f_src", "f_dst", "i_src", "i_dst")}
        r.update({k: np.empty(V, np.uint32) for k in ("f_outdeg", "f_indeg", "f_idx", "i_outdeg", "i_indeg",
                                                        "i_idx")})
        if w is not None:
            r["f_w"], r["i_w"] = np.empty(E, np.float32), np.empty(E, np.float32)
        st = self.d.orc_build(E, V, _p(src), _p(dst), _p(w), sort_type, _p(r["f_src"]), _p(r["f_dst"]),
                              _p(r.get("f_w")), _p(r["f_outdeg"]), _p(r["f_indeg"]), _p(r["f_idx"]),
                              _p(r["i_src"]), _p(r["i_dst"]), _p(r.get("i_w")), _p(r["i_outdeg"]),
                              _p(r["i_indeg"]), _p(r["i_idx"]))
        if st:
            raise ValueError("oracle build: an id is >= V")
        r["num_vertices"], r["num_edges"] = V, E
        return r

    def dedup(self, s, d, w=None, truncate_w: bool = False):
        E = len(s)
        os_, od = np.empty(E, np.uint32), np.empty(E, np.uint32)
        ow = np.empty(E, np.float32) if w is not None else None
        n = self.d.orc_dedup(E, _p(s), _p(d), _p(w), _p(os_), _p(od), _p(ow), 1 if truncate_w else 0)
        return os_[:n], od[:n], (ow[:n] if ow is not None else None)

    def bfs(self, g: dict, root: int, mode: int = 2, bitmap_nf: bool = False):
        V, E = g["num_vertices"], g["num_edges"]
        par, dist = np.empty(V, np.int32), np.empty(V, np.uint32)

        class St(C.Structure):
            _fields_ = [("iteration", u32), ("processed_nodes", u32), ("td_steps", u32), ("bu_steps", u32),
                        ("reached", u32), ("reached_out_edges", C.c_uint64)]
        st = St()
        dirs = np.zeros(4096, np.uint8)
        r = self.d.orc_bfs(V, E, _p(g["f_outdeg"]), _p(g["f_idx"]), _p(g["f_dst"]), _p(g["i_outdeg"]),
                           _p(g["i_idx"]), _p(g["i_dst"]), root, mode, 1 if bitmap_nf else 0, _p(par), _p(dist),
                           C.addressof(st), _p(dirs), len(dirs))
        if r:
            raise ValueError("oracle bfs: bad root")
        stats = {f: getattr(st, f) for f, _ in St._fields_}
        nsteps = stats["td_steps"] + stats["bu_steps"]
        stats["dirs"] = dirs[:min(nsteps, len(dirs))].copy()
        return par, dist, stats

    def pagerank(self, g: dict, mode: int = 0, max_iters: int = 20, epsilon: float = 1e-4, init=None):
        V = g["num_vertices"]
        ranks = np.empty(V, np.float32)
        it, err = u32(), C.c_double()
        eh = np.zeros(max(max_iters, 1), np.float64)
        ah = np.zeros(max(max_iters, 1), np.uint32)
        n = self.d.orc_pagerank(V, _p(g["f_outdeg"]), _p(g["f_idx"]), _p(g["f_dst"]), _p(g["i_outdeg"]),
                                _p(g["i_idx"]), _p(g["i_dst"]), mode, max_iters, epsilon, _p(init), _p(ranks),
                                C.byref(it), C.byref(err), _p(eh), _p(ah))
        return ranks, {"iterations": it.value, "error_total": err.value, "executed": n, "err_hist": eh[:n],
                       "active_hist": ah[:n]}

    def pagerank_f64(self, g: dict, iters: int, init=None):
        V = g["num_vertices"]
        ranks = np.empty(V, np.float64)
        self.d.orc_pagerank_f64(V, _p(g["f_outdeg"]), _p(g["i_outdeg"]), _p(g["i_idx"]), _p(g["i_dst"]), iters,
                                _p(init), _p(ranks))
        return ranks

    @staticmethod
    def ppr_f64(g: dict, seeds, iters: int, damp: float = 0.85):
        """Personalized PageRank in FP64, one vector per seed, as a restatement
        of the reference's pull iteration (pageRank.c:984-1044) with the
        teleport term base_pr replaced by (1 - damp) on the seed vertex only,
        started from the seed's one-hot vector; dangling rank is not
        redistributed (as in the reference).  Returns (ranks [V, S], the L1
        change of each vector per iteration [iters, S]).  Numpy, small graphs."""
        V = g["num_vertices"]
        outdeg = g["f_outdeg"].astype(np.float64)
        idx, deg, nbr = g["i_idx"].astype(np.int64), g["i_outdeg"].astype(np.int64), g["i_dst"].astype(np.int64)
        # destination of every inverse edge, in CSR order
        dst = np.repeat(np.arange(V), deg)
        src = np.concatenate([nbr[idx[v]: idx[v] + deg[v]] for v in range(V)]) if len(dst) else np.zeros(0, np.int64)
        S = len(seeds)
        r = np.zeros((V, S))
        r[np.asarray(seeds), np.arange(S)] = 1.0
        tele = np.zeros((V, S))
        tele[np.asarray(seeds), np.arange(S)] = 1.0 - damp
        inv = np.where(outdeg > 0, 1.0 / np.maximum(outdeg, 1), 0.0)
        hist = np.zeros((iters, S))
        for it in range(iters):
            c = r * inv[:, None]
            s = np.zeros((V, S))
            np.add.at(s, dst, c[src])
            nr = tele + damp * s
            hist[it] = np.abs(nr - r).sum(axis=0)
            r = nr
        return r, hist

    def random_roots(self, V: int, avg_degree: int, out_degree, n: int, seed: int = 27491095):
        roots = np.empty(n, np.uint32)
        self.d.orc_random_roots(seed, V, avg_degree, _p(out_degree), n, _p(roots))
        return roots


def write_edge_file(path: str, src, dst, w=None) -> None:
    """The reference's binary edge file (edgeList.c:336-594): little-endian
    {u32 src, u32 dst} records (.bin), or {u32 src, u32 dst, f32 w} (.wbin)."""
    rec = np.empty((len(src), 3 if w is not None else 2), np.uint32)
    rec[:, 0] = src
    rec[:, 1] = dst
    if w is not None:
        rec[:, 2] = np.asarray(w, np.float32).view(np.uint32)
    rec.astype("<u4", copy=False).tofile(path)


@contextlib.contextmanager
def silenced_stdout():
    """Send the C library's stdout (fd 1) to /dev/null for the duration."""
    libc = C.CDLL(None)
    libc.fflush(None)
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


class Reference:
    """The reference's own CPU build (oracle/_ref), bound with the same struct
    layouts as the product (layouts checked by tests/test_abi.py)."""

    def __init__(self, weighted: bool = False):
        import opengraph_b200 as og
        self.og = og
        self.weighted = weighted
        path = os.path.join(REF_DIR, "libogref_w.so" if weighted else "libogref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.d = C.CDLL(path)
        EL = og.EdgeListW if weighted else og.EdgeList
        G = og.GraphCSRW if weighted else og.GraphCSR
        self.EdgeList, self.GraphCSR = EL, G
        for name, res, args in og._api(EL, G):
            if hasattr(self.d, name):
                fn = getattr(self.d, name)
                fn.restype, fn.argtypes = res, args
                setattr(self, name, fn)

    @staticmethod
    def available(weighted: bool = False) -> bool:
        return os.path.exists(os.path.join(REF_DIR, "libogref_w.so" if weighted else "libogref.so"))

    def arguments(self, **kw):
        a = self.og.default_arguments(**kw)
        self.initializeMersenneState(C.byref(a.mt19937var), 27491095)
        return a

    def build_graph(self, path: str, sort: int = 0, dflag: int = 0, weighted_file: bool = False, quiet=True):
        a = self.arguments(fnameb=path, sort=sort, dflag=dflag, weighted=1 if weighted_file else 0)
        self._keep = a
        with (silenced_stdout() if quiet else contextlib.nullcontext()):
            g = self.graphCSRPreProcessingStep(C.byref(a))
        return g

    def bfs(self, g, root: int, pushpull: int = 2, quiet=True):
        a = self.arguments(source=root, pushpull=pushpull)
        with (silenced_stdout() if quiet else contextlib.nullcontext()):
            st = self.breadthFirstSearchGraphCSR(C.byref(a), g)
        s = st.contents
        V = s.num_vertices
        out = (self.og.as_numpy(s.parents, V, np.int32), self.og.as_numpy(s.distances, V, np.uint32),
               {"processed_nodes": s.processed_nodes, "iteration": s.iteration, "time_total": s.time_total})
        self.freeBFSStats(st)
        return out

    def pagerank(self, g, pushpull: int = 0, iterations: int = 20, epsilon: float = 1e-4, quiet=True):
        a = self.arguments(pushpull=pushpull, iterations=iterations, epsilon=epsilon)
        with (silenced_stdout() if quiet else contextlib.nullcontext()):
            st = self.pageRankGraphCSR(C.byref(a), g)
        s = st.contents
        V = s.num_vertices
        out = (self.og.as_numpy(s.pageRanks, V, np.float32),
               {"iterations": s.iterations, "error_total": s.error_total, "time_total": s.time_total})
        self.freePageRankStats(st)
        return out
