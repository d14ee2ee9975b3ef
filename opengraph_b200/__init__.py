"""B200-native OpenGraph CSR hot path (sort + CSR build, PageRank, DO-BFS).

The product is the C-ABI library ``libogb200.so`` (WEIGHTED=0 layout) /
``libogb200_w.so`` (WEIGHTED=1), built in-tree by ``opengraph_b200.build``.
This module binds it with ctypes:

* ``Library.<reference name>`` -- the OpenGraph C API (``include/ogb200.h``),
  same names, arguments and struct layouts as OpenGraph's
  ``graphCSRPreProcessingStep``, ``sortRunAlgorithms``,
  ``breadthFirstSearchGraphCSR``, ``pageRankGraphCSR`` ...;
* ``Library.device_graph`` / ``DeviceGraph`` -- the status-returning device
  API (``include/ogb200_device.h``) over torch CUDA tensors.

There is no CPU fallback: loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAMES = {False: "libogb200.so", True: "libogb200_w.so"}

u32 = C.c_uint32
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
f32p = C.POINTER(C.c_float)
vp = C.c_void_p


# ----------------------------------------------------------------- structs --

class mt19937state(C.Structure):
    """00_graph_bench/include/utils/mt19937.h:38-44"""
    _fields_ = [("mt", C.c_ulong * 624), ("mti", C.c_int)]


class Arguments(C.Structure):
    """00_graph_bench/include/config/graphConfig.h:11-44"""
    _fields_ = [
        ("wflag", C.c_int), ("xflag", C.c_int), ("sflag", C.c_int), ("Sflag", C.c_int), ("dflag", C.c_int),
        ("binSize", u32), ("verbosity", u32), ("iterations", u32), ("trials", u32), ("epsilon", C.c_double),
        ("source", C.c_int), ("algorithm", u32), ("datastructure", u32), ("pushpull", u32), ("sort", u32),
        ("lmode", u32), ("lmode_l2", u32), ("lmode_l3", u32), ("mmode", u32), ("symmetric", u32),
        ("weighted", u32), ("delta", u32), ("pre_numThreads", C.c_int), ("algo_numThreads", C.c_int),
        ("ker_numThreads", C.c_int), ("fnameb", C.c_char_p), ("fnamel", C.c_char_p), ("fnameb_format", u32),
        ("convert_format", u32), ("mt19937var", mt19937state), ("cache_size", u32),
    ]


class Vertex(C.Structure):
    """00_graph_bench/include/structures/vertex.h:13-18"""
    _fields_ = [("out_degree", u32p), ("in_degree", u32p), ("edges_idx", u32p)]


class EdgeList(C.Structure):
    """edgeList.h:8-23, WEIGHTED=0"""
    _fields_ = [("num_edges", u32), ("num_vertices", u32), ("avg_degree", u32), ("edges_array_src", u32p),
                ("edges_array_dest", u32p), ("mask_array", u32p), ("label_array", u32p),
                ("inverse_label_array", u32p)]


class EdgeListW(C.Structure):
    """edgeList.h:8-23, WEIGHTED=1"""
    _fields_ = [("num_edges", u32), ("num_vertices", u32), ("avg_degree", u32), ("max_weight", C.c_float),
                ("edges_array_weight", f32p), ("edges_array_src", u32p), ("edges_array_dest", u32p),
                ("mask_array", u32p), ("label_array", u32p), ("inverse_label_array", u32p)]


class GraphCSR(C.Structure):
    """graphCSR.h:12-29, WEIGHTED=0, DIRECTED=1"""
    _fields_ = [("num_edges", u32), ("num_vertices", u32), ("avg_degree", u32), ("vertices", C.POINTER(Vertex)),
                ("sorted_edges_array", C.POINTER(EdgeList)), ("inverse_vertices", C.POINTER(Vertex)),
                ("inverse_sorted_edges_array", C.POINTER(EdgeList))]


class GraphCSRW(C.Structure):
    """graphCSR.h:12-29, WEIGHTED=1, DIRECTED=1"""
    _fields_ = [("num_edges", u32), ("num_vertices", u32), ("avg_degree", u32), ("max_weight", C.c_float),
                ("vertices", C.POINTER(Vertex)), ("sorted_edges_array", C.POINTER(EdgeListW)),
                ("inverse_vertices", C.POINTER(Vertex)), ("inverse_sorted_edges_array", C.POINTER(EdgeListW))]


class BFSStats(C.Structure):
    """algorithms/openmp/BFS.h:19-29"""
    _fields_ = [("distances", u32p), ("parents", i32p), ("distances_DualOrder", u32p), ("parents_DualOrder", i32p),
                ("processed_nodes", u32), ("num_vertices", u32), ("iteration", u32), ("time_total", C.c_double)]


class PageRankStats(C.Structure):
    """algorithms/openmp/pageRank.h:19-30"""
    _fields_ = [("damp", C.c_float), ("base_pr", C.c_float), ("iterations", u32), ("num_vertices", u32),
                ("activeVertices", u32), ("realRanks", u32p), ("pageRanks", f32p), ("time_total", C.c_double),
                ("error_total", C.c_double)]


class SPMVStats(C.Structure):
    """algorithms/openmp/SPMV.h:19-27"""
    _fields_ = [("iterations", u32), ("arguments", vp), ("num_vertices", u32), ("vector_output", f32p),
                ("vector_input", f32p), ("time_total", C.c_double)]


class Bitmap(C.Structure):
    """structures/bitmap.h:19-26"""
    _fields_ = [("real_size", u32), ("size", u32), ("numSetBits", u32), ("bitarray", u32p)]


class ArrayQueue(C.Structure):
    """structures/arrayQueue.h:7-16"""
    _fields_ = [("head", u32), ("tail", u32), ("tail_next", u32), ("size", u32), ("queue", u32p),
                ("q_bitmap", C.POINTER(Bitmap)), ("q_bitmap_next", C.POINTER(Bitmap))]


# ---------------------------------------------------------- device structs --

class CsrView(C.Structure):
    _fields_ = [("num_vertices", u32), ("num_edges", u32), ("src", vp), ("dst", vp), ("weight", vp),
                ("out_degree", vp), ("in_degree", vp), ("edges_idx", vp)]


class BfsInfo(C.Structure):
    _fields_ = [("iteration", u32), ("processed_nodes", u32), ("td_steps", u32), ("bu_steps", u32),
                ("reached", u32), ("levels", u32), ("reached_out_edges", C.c_uint64),
                ("edges_examined", C.c_uint64), ("ms", C.c_double), ("launches", u32), ("pad", u32)]


class MsBfsInfo(C.Structure):
    _fields_ = [("levels", u32), ("push_levels", u32), ("pull_levels", u32), ("launches", u32),
                ("reached_pairs", C.c_uint64), ("edges_examined", C.c_uint64), ("ms", C.c_double),
                ("init_ms", C.c_double)]


class PprBatchInfo(C.Structure):
    _fields_ = [("executed", u32), ("converged", u32), ("launches", u32), ("pad", u32), ("ms", C.c_double),
                ("err_last", C.c_double * 32)]


class BatchBfsInfo(C.Structure):
    _fields_ = [("levels", u32), ("td_steps", u32), ("bu_steps", u32), ("reached", u32), ("ms", C.c_double)]


class BatchPrGraph(C.Structure):
    _fields_ = [("iterations", u32), ("executed", u32), ("activeVertices", u32), ("converged", u32),
                ("error_total", C.c_double)]


class BatchPrInfo(C.Structure):
    _fields_ = [("ms", C.c_double), ("captured", u32), ("pad", u32)]


class TuneInfo(C.Structure):
    _fields_ = [("ncandidates", u32), ("best", u32), ("warp_thr", u32 * 16), ("cta_thr", u32 * 16),
                ("ms", C.c_double * 16)]


class BfsLevel(C.Structure):
    _fields_ = [("direction", u32), ("discovered", u32), ("frontier", u32), ("mf", u32), ("mu", u32),
                ("pad", u32), ("edges", C.c_uint64), ("ms", C.c_float), ("pad2", C.c_float)]


class SpmvInfo(C.Structure):
    _fields_ = [("iterations", u32), ("weighted", u32), ("ms", C.c_double)]


class PrInfo(C.Structure):
    _fields_ = [("iterations", u32), ("executed", u32), ("activeVertices", u32), ("converged", u32),
                ("error_total", C.c_double), ("ms", C.c_double), ("launches", u32), ("pad", u32)]


def info_dict(s: C.Structure) -> dict:
    return {f: getattr(s, f) for f, _ in s._fields_ if not f.startswith("pad")}


# ------------------------------------------------------------------ library --

# (name, restype, argtypes) of the OpenGraph C API, filled per layout
def _api(EL, G):
    ELp, Gp = C.POINTER(EL), C.POINTER(G)
    Ap = C.POINTER(Arguments)
    return [
        ("readEdgeListsbin", ELp, [C.c_char_p, C.c_uint8, u32, u32]),
        ("readEdgeListsMem", ELp, [ELp, C.c_uint8, u32, u32]),
        ("newEdgeList", ELp, [u32]),
        ("freeEdgeList", None, [ELp]),
        ("removeDulpicatesSelfLoopEdges", ELp, [ELp]),
        ("sortRunAlgorithms", ELp, [ELp, u32]),
        ("radixSortEdgesBySource", ELp, [ELp]),
        ("radixSortEdgesBySourceAndDestination", ELp, [ELp]),
        ("countSortEdgesBySource", ELp, [ELp]),
        ("countSortEdgesByDestination", ELp, [ELp]),
        ("countSortEdgesBySourceAndDestination", ELp, [ELp]),
        ("newVertexArray", C.POINTER(Vertex), [u32]),
        ("freeVertexArray", None, [C.POINTER(Vertex)]),
        ("mapVerticesWithInOutDegree", Gp, [Gp, C.c_uint8]),
        ("graphCSRNew", Gp, [u32, u32, C.c_uint8]),
        ("graphCSRAssignEdgeList", Gp, [Gp, ELp, C.c_uint8]),
        ("graphCSRPreProcessingStep", Gp, [Ap]),
        ("graphCSRFree", None, [Gp]),
        ("graphCSRPrint", None, [Gp]),
        ("newBFSStatsGraphCSR", C.POINTER(BFSStats), [Gp]),
        ("freeBFSStats", None, [C.POINTER(BFSStats)]),
        ("breadthFirstSearchGraphCSR", C.POINTER(BFSStats), [Ap, Gp]),
        ("breadthFirstSearchPullGraphCSR", C.POINTER(BFSStats), [Ap, Gp]),
        ("breadthFirstSearchPushGraphCSR", C.POINTER(BFSStats), [Ap, Gp]),
        ("breadthFirstSearchDirectionOptimizedGraphCSR", C.POINTER(BFSStats), [Ap, Gp]),
        ("breadthFirstSearchPushBitmapGraphCSR", C.POINTER(BFSStats), [Ap, Gp]),
        ("breadthFirstSearchPushDirectionOptimizedBitmapGraphCSR", C.POINTER(BFSStats), [Ap, Gp]),
        ("topDownStepGraphCSR", u32, [Gp, C.POINTER(ArrayQueue), C.POINTER(C.POINTER(ArrayQueue)),
                                      C.POINTER(BFSStats)]),
        ("bottomUpStepGraphCSR", u32, [Gp, C.POINTER(Bitmap), C.POINTER(Bitmap), C.POINTER(BFSStats)]),
        ("readFromBinFileGraphCSR", Gp, [C.c_char_p]),
        ("writeToBinFileGraphCSR", None, [C.c_char_p, Gp]),
        ("graphCSRPreProcessingStepDualOrder", Gp, [Ap]),
        ("graphCSRVertexLabelRemappingDualOrder", None, [Gp]),
        ("breadthFirstSearchGraphCSRDualOrder", C.POINTER(BFSStats), [Ap, Gp]),
        ("breadthFirstSearchPullGraphCSRDualOrder", C.POINTER(BFSStats), [Ap, Gp]),
        ("breadthFirstSearchPushGraphCSRDualOrder", C.POINTER(BFSStats), [Ap, Gp]),
        ("breadthFirstSearchDirectionOptimizedGraphCSRDualOrder", C.POINTER(BFSStats), [Ap, Gp]),
        ("topDownStepGraphCSRDualOrder", u32, [Gp, C.POINTER(ArrayQueue), C.POINTER(C.POINTER(ArrayQueue)),
                                               C.POINTER(BFSStats)]),
        ("bottomUpStepGraphCSRDualOrder", u32, [Gp, C.POINTER(Bitmap), C.POINTER(Bitmap), C.POINTER(BFSStats)]),
        ("newPageRankStatsGraphCSR", C.POINTER(PageRankStats), [Gp]),
        ("freePageRankStats", None, [C.POINTER(PageRankStats)]),
        ("pageRankGraphCSR", C.POINTER(PageRankStats), [Ap, Gp]),
        ("pageRankPullGraphCSR", C.POINTER(PageRankStats), [Ap, Gp]),
        ("pageRankPushGraphCSR", C.POINTER(PageRankStats), [Ap, Gp]),
        ("pageRankDataDrivenPullGraphCSR", C.POINTER(PageRankStats), [Ap, Gp]),
        ("pageRankDataDrivenPushGraphCSR", C.POINTER(PageRankStats), [Ap, Gp]),
        ("pageRankDataDrivenPullPushGraphCSR", C.POINTER(PageRankStats), [Ap, Gp]),
        ("radixSortEdgesByPageRank", u32p, [f32p, u32p, u32]),
        ("newSPMVStatsGraphCSR", C.POINTER(SPMVStats), [Gp]),
        ("freeSPMVStats", None, [C.POINTER(SPMVStats)]),
        ("SPMVGraphCSR", C.POINTER(SPMVStats), [Ap, Gp]),
        ("SPMVPullGraphCSR", C.POINTER(SPMVStats), [Ap, Gp]),
        ("SPMVPushGraphCSR", C.POINTER(SPMVStats), [Ap, Gp]),
        ("initializeMersenneState", None, [C.POINTER(mt19937state), C.c_ulong]),
        ("generateRandInt", C.c_ulong, [C.POINTER(mt19937state)]),
        ("generateRandFloat", C.c_float, [C.POINTER(mt19937state)]),
        ("generateRandomRootGraphCSR", u32, [C.POINTER(mt19937state), Gp]),
    ]


_DEVICE_API = [
    ("ogb_last_error", C.c_char_p, []),
    ("ogb_weighted_layout", C.c_int, []),
    ("ogb_set_quiet", None, [C.c_int]),
    ("ogb_dropin_bfs_phases", C.c_int, [C.POINTER(C.c_double), u32]),
    ("ogb_graph_create", C.c_int, [C.POINTER(vp)]),
    ("ogb_graph_destroy", None, [vp]),
    ("ogb_graph_build", C.c_int, [vp, vp, vp, vp, u32, u32, u32, vp]),
    ("ogb_graph_view", C.c_int, [vp, C.c_int, C.POINTER(CsrView)]),
    ("ogb_graph_of", vp, [vp]),
    ("ogb_sort_edges", C.c_int, [vp, vp, vp, u32, u32, vp, vp, vp, vp]),
    ("ogb_bfs", C.c_int, [vp, u32, u32, vp, vp, C.POINTER(BfsInfo), vp]),
    ("ogb_bfs_trace", C.c_int, [vp, C.POINTER(BfsLevel), u32, C.POINTER(u32)]),
    ("ogb_msbfs", C.c_int, [vp, u32p, u32, vp, C.POINTER(MsBfsInfo), vp]),
    ("ogb_bfs_features", C.c_int, [vp, vp, u32, C.POINTER(u32)]),
    ("ogb_bfs_set_policy", C.c_int, [vp]),
    ("ogb_mlp_nparams", u32, [u32, u32]),
    ("ogb_mlp_grad", C.c_int, [u32, u32, u32, vp, vp, u32, vp, vp, C.POINTER(C.c_float), vp]),
    ("ogb_mlp_train", C.c_int, [u32, u32, u32, vp, vp, u32, u32, u32, C.c_float, u32, vp, vp, vp]),
    ("ogb_mlp_infer", C.c_int, [u32, u32, vp, vp, u32, vp, vp]),
    ("ogb_pagerank_warm_start", C.c_int, [vp, u32, vp, vp, vp]),
    ("ogb_ppr", C.c_int, [vp, u32p, u32, u32, C.c_double, vp, C.POINTER(PprBatchInfo), vp]),
    ("ogb_batch_create", vp, [u32, u32p, C.POINTER(C.c_uint64), u32p, u32p, u32]),
    ("ogb_batch_free", None, [vp]),
    ("ogb_batch_offsets", C.c_int, [vp, u32p]),
    ("ogb_batch_bfs", C.c_int, [vp, u32p, vp, vp, C.POINTER(BatchBfsInfo), vp]),
    ("ogb_batch_pagerank", C.c_int, [vp, u32, C.c_double, vp, vp, C.POINTER(BatchPrInfo), vp]),
    ("ogb_batch_autotune", C.c_int, [vp, C.POINTER(TuneInfo)]),
    ("ogb_pagerank", C.c_int, [vp, u32, u32, C.c_double, vp, vp, C.POINTER(PrInfo), vp]),
    ("ogb_pagerank_history", C.c_int, [vp, C.POINTER(C.c_double), u32p, u32, C.POINTER(u32)]),
    ("ogb_spmv", C.c_int, [vp, u32, u32, vp, vp, C.POINTER(SpmvInfo), vp]),
    ("ogb_sort_by_rank", C.c_int, [vp, vp, u32, vp]),
    ("ogb_pagerank_range_init", C.c_int, [vp, vp, vp, vp]),
    ("ogb_pagerank_range_step", C.c_int, [vp, u32, u32, vp, vp, vp, C.c_double, vp, vp, vp]),
    ("ogb_pagerank_range_finish", C.c_int, [vp, vp, vp]),
    ("ogb_pagerank_range_step_peers", C.c_int, [vp, u32, u32, vp, vp, vp, vp, u32, C.c_double, vp, vp, vp]),
    ("ogb_partition_edges", C.c_int, [vp, vp, vp, u32, vp, u32, vp, vp, vp, vp, vp]),
    ("ogb_bfs_range_expand_peers", C.c_int, [vp, u32, u32, u32, u32, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp]),
    ("ogb_bfs_range_claim_peers", C.c_int, [vp, u32, u32, u32, u32, vp, vp, vp, u32, vp, vp, vp, vp]),
    ("ogb_bfs_range_init", C.c_int, [vp, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp]),
    ("ogb_bfs_range_expand", C.c_int, [vp, u32, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp]),
    ("ogb_bfs_range_settle", C.c_int, [vp, u32, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp]),
    ("ogb_pagerank_set_bins", None, [u32, u32]),
    ("ogb_pagerank_pull_noalloc", C.c_int, [u32, vp, vp, vp, vp, u32, C.c_double, vp, vp, vp]),
    ("ogb_pagerank_get_bins", None, [u32p, u32p, u32p, u32p]),
    ("ogb_generate_rmat", C.c_int, [u32, u32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_int, vp, vp,
                                    vp]),
    ("ogb_generate_uniform", C.c_int, [u32, C.c_uint64, C.c_uint64, vp, vp, vp]),
    ("ogb_generate_grid", C.c_int, [u32, C.c_double, C.c_uint64, vp, vp, vp, C.POINTER(C.c_uint64)]),
    ("ogb_write_edge_file", C.c_int, [C.c_char_p, vp, vp, vp, C.c_uint64]),
]


class OgbError(RuntimeError):
    pass


def lib_path(weighted: bool = False) -> str:
    return os.path.join(HERE, LIB_NAMES[bool(weighted)])


class Library:
    """One loaded layout of libogb200 (weighted=False: WEIGHTED=0)."""

    def __init__(self, weighted: bool = False, path: str | None = None):
        self.weighted = bool(weighted)
        self.path = path or lib_path(weighted)
        if not os.path.exists(self.path):
            raise OgbError(f"{self.path} is missing: build it with `python -m opengraph_b200.build`")
        self.dll = C.CDLL(self.path)
        self.EdgeList = EdgeListW if self.weighted else EdgeList
        self.GraphCSR = GraphCSRW if self.weighted else GraphCSR
        for name, res, args in _api(self.EdgeList, self.GraphCSR) + _DEVICE_API:
            fn = getattr(self.dll, name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)
        if self.ogb_weighted_layout() != int(self.weighted):
            raise OgbError(f"{self.path}: layout mismatch")

    # -- helpers -------------------------------------------------------------
    def check(self, status: int, what: str = "") -> None:
        if status != 0:
            msg = self.ogb_last_error()
            raise OgbError(f"{what} failed with status {status}: {msg.decode() if msg else ''}")

    def quiet(self, q: bool = True) -> None:
        self.ogb_set_quiet(1 if q else 0)

    def device_graph(self) -> "DeviceGraph":
        return DeviceGraph(self)


_LIBS: dict[bool, Library] = {}


def load(weighted: bool = False) -> Library:
    """The process-wide Library for a layout (loaded once)."""
    w = bool(weighted)
    if w not in _LIBS:
        _LIBS[w] = Library(w)
    return _LIBS[w]


def mlp_nparams(lib, n_in: int, hidden: int) -> int:
    return int(lib.ogb_mlp_nparams(n_in, hidden))


def mlp_init(lib, n_in: int, hidden: int, seed: int = 0) -> np.ndarray:
    """He-initialized fp32 parameters in the library's packing."""
    rng = np.random.default_rng(seed)
    p = np.zeros(mlp_nparams(lib, n_in, hidden), np.float32)
    o = 0
    for fan_in, n_out in ((n_in, hidden), (hidden, hidden), (hidden, 1)):
        w = rng.normal(0.0, np.sqrt(2.0 / fan_in), size=(n_out, fan_in)).astype(np.float32)
        p[o: o + w.size] = w.ravel()
        o += w.size + n_out  # biases start at 0
    return p


def mlp_grad(lib, n_in, hidden, loss, X, T, params, stream=None):
    """Batch-mean loss and gradient (device tensors X [B, in], T [B])."""
    g = np.zeros_like(params)
    l = C.c_float()
    lib.check(lib.ogb_mlp_grad(n_in, hidden, loss, _ptr(X), _ptr(T), int(T.numel()), params.ctypes.data, g.ctypes.data,
                               C.byref(l), _stream(stream)), "ogb_mlp_grad")
    return l.value, g


def mlp_train(lib, n_in, hidden, loss, X, T, params, epochs=10, batch=4096, lr=1e-3, seed=0, stream=None):
    p = np.ascontiguousarray(params.astype(np.float32).copy())
    hist = np.zeros(max(epochs, 1), np.float32)
    lib.check(lib.ogb_mlp_train(n_in, hidden, loss, _ptr(X), _ptr(T), int(T.numel()), epochs, batch, float(lr), seed,
                                p.ctypes.data, hist.ctypes.data, _stream(stream)), "ogb_mlp_train")
    return p, hist[:epochs]


def mlp_infer(lib, n_in, hidden, params, X, Y, stream=None):
    p = np.ascontiguousarray(np.asarray(params, np.float32))
    lib.check(lib.ogb_mlp_infer(n_in, hidden, p.ctypes.data, _ptr(X), int(Y.numel()), _ptr(Y), _stream(stream)),
              "ogb_mlp_infer")


def default_arguments(**overrides) -> Arguments:
    """struct Arguments with the reference CLI defaults (open-graph.c:273-305);
    the MT19937 state is seeded by the caller's library (seed 27491095)."""
    a = Arguments()
    a.binSize, a.iterations, a.trials, a.epsilon = 512, 20, 1, 0.0001
    a.cache_size, a.delta = 32768, 1
    nt = os.cpu_count() or 1
    a.pre_numThreads = a.algo_numThreads = a.ker_numThreads = nt
    a.fnameb_format = a.convert_format = 1
    for k, v in overrides.items():
        if k == "fnameb" and isinstance(v, str):
            v = v.encode()
        setattr(a, k, v)
    return a


# ----------------------------------------------------------- numpy views --

def as_numpy(ptr, n: int, dtype) -> np.ndarray:
    """Copy n elements behind a ctypes pointer into a numpy array."""
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def edge_list_arrays(el) -> dict:
    e = el.contents
    d = {"src": as_numpy(e.edges_array_src, e.num_edges, np.uint32),
         "dst": as_numpy(e.edges_array_dest, e.num_edges, np.uint32),
         "num_vertices": e.num_vertices, "num_edges": e.num_edges, "avg_degree": e.avg_degree}
    if hasattr(e, "edges_array_weight"):
        d["w"] = as_numpy(e.edges_array_weight, e.num_edges, np.float32)
        d["max_weight"] = e.max_weight
    return d


def graph_arrays(g) -> dict:
    h = g.contents
    V = h.num_vertices
    out = {"num_vertices": V, "num_edges": h.num_edges, "avg_degree": h.avg_degree}
    for tag, verts, el in (("f", h.vertices, h.sorted_edges_array), ("i", h.inverse_vertices,
                                                                       h.inverse_sorted_edges_array)):
        v = verts.contents
        out[tag + "_outdeg"] = as_numpy(v.out_degree, V, np.uint32)
        out[tag + "_indeg"] = as_numpy(v.in_degree, V, np.uint32)
        out[tag + "_idx"] = as_numpy(v.edges_idx, V, np.uint32)
        ea = edge_list_arrays(el)
        out[tag + "_src"], out[tag + "_dst"] = ea["src"], ea["dst"]
        if "w" in ea:
            out[tag + "_w"] = ea["w"]
    return out


# ------------------------------------------------------------ device graph --

def _ptr(t) -> int | None:
    if t is None:
        return None
    return int(t.data_ptr())


_CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the legacy default stream


def _stream(stream) -> int:
    """The stream a call runs on: the caller's, else torch's current stream
    (so the call is ordered after the torch work that filled its inputs; the
    legacy default stream is passed as cudaStreamLegacy)."""
    if stream is not None:
        return int(stream)
    import torch
    h = int(torch.cuda.current_stream().cuda_stream)
    return h if h else _CUDA_STREAM_LEGACY


class _CudaArray:
    """Zero-copy __cuda_array_interface__ view of library-owned device memory."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None}


@dataclass
class CsrArrays:
    num_vertices: int
    num_edges: int
    src: object
    dst: object
    weight: object
    out_degree: object
    in_degree: object
    edges_idx: object


class GraphBatch:
    """Many graphs packed into one device union (ogb_batch_*): edge lists in
    local ids, back to back; every vertex array of the batch holds the
    graphs' vertices back to back (offsets)."""

    def __init__(self, lib, num_vertices, edge_offsets, src, dst, sort_type: int = 0):
        self.lib = lib
        nv = np.ascontiguousarray(np.asarray(num_vertices, dtype=np.uint32))
        eo = np.ascontiguousarray(np.asarray(edge_offsets, dtype=np.uint64))
        s = np.ascontiguousarray(np.asarray(src, dtype=np.uint32))
        d = np.ascontiguousarray(np.asarray(dst, dtype=np.uint32))
        self.n = len(nv)
        h = lib.ogb_batch_create(self.n, nv.ctypes.data_as(u32p), eo.ctypes.data_as(C.POINTER(C.c_uint64)),
                                 s.ctypes.data_as(u32p), d.ctypes.data_as(u32p), int(sort_type))
        if not h:
            msg = lib.ogb_last_error()
            raise OgbError("ogb_batch_create: " + (msg.decode() if msg else ""))
        self.handle = h
        off = np.zeros(self.n + 1, np.uint32)
        lib.check(lib.ogb_batch_offsets(h, off.ctypes.data_as(u32p)), "ogb_batch_offsets")
        self.offsets = off

    def bfs(self, roots, parents, distances, stream=None) -> dict:
        r = np.ascontiguousarray(np.asarray(roots, dtype=np.uint32))
        info = BatchBfsInfo()
        self.lib.check(self.lib.ogb_batch_bfs(self.handle, r.ctypes.data_as(u32p), _ptr(parents), _ptr(distances),
                                              C.byref(info), _stream(stream)), "ogb_batch_bfs")
        return info_dict(info)

    def pagerank(self, ranks, max_iterations: int = 100, epsilon: float = 1e-4, stream=None):
        per = (BatchPrGraph * self.n)()
        info = BatchPrInfo()
        self.lib.check(self.lib.ogb_batch_pagerank(self.handle, int(max_iterations), float(epsilon), _ptr(ranks),
                                                   per, C.byref(info), _stream(stream)), "ogb_batch_pagerank")
        return info_dict(info), [info_dict(per[i]) for i in range(self.n)]

    def autotune(self) -> dict:
        t = TuneInfo()
        self.lib.check(self.lib.ogb_batch_autotune(self.handle, C.byref(t)), "ogb_batch_autotune")
        n = t.ncandidates
        return {"best": t.best, "candidates": [(t.warp_thr[i], t.cta_thr[i], t.ms[i]) for i in range(n)]}

    def close(self):
        if self.handle:
            self.lib.ogb_batch_free(self.handle)
            self.handle = None


class DeviceGraph:
    """Device-resident CSR (both directions) built by the library's kernels."""

    def __init__(self, lib: Library, handle: int | None = None, owned: bool = True):
        self.lib = lib
        self.owned = owned
        if handle is None:
            h = vp()
            lib.check(lib.ogb_graph_create(C.byref(h)), "ogb_graph_create")
            handle = h.value
        self.handle = handle

    def close(self) -> None:
        if self.handle and self.owned:
            self.lib.ogb_graph_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, src, dst, num_vertices: int, sort_type: int = 0, weight=None, stream=None) -> None:
        """Sort + CSR build from device tensors (uint32 viewed as int32 is fine)."""
        self.lib.check(self.lib.ogb_graph_build(self.handle, _ptr(src), _ptr(dst), _ptr(weight), int(src.numel()),
                                                int(num_vertices), int(sort_type), _stream(stream)), "ogb_graph_build")

    def view(self, inverse: bool = False) -> CsrArrays:
        """Zero-copy torch views of one direction's device arrays."""
        import torch
        v = CsrView()
        self.lib.check(self.lib.ogb_graph_view(self.handle, 1 if inverse else 0, C.byref(v)), "ogb_graph_view")
        V, E = v.num_vertices, v.num_edges

        def t(ptr, n, ts):
            if not ptr or n == 0:
                return None
            return torch.as_tensor(_CudaArray(ptr, n, ts), device="cuda")
        return CsrArrays(V, E, t(v.src, E, "<i4"), t(v.dst, E, "<i4"), t(v.weight, E, "<f4"),
                         t(v.out_degree, V, "<i4"), t(v.in_degree, V, "<i4"), t(v.edges_idx, V, "<i4"))

    def bfs(self, root: int, parents, distances, mode: int = 2, stream=None) -> dict:
        info = BfsInfo()
        self.lib.check(self.lib.ogb_bfs(self.handle, int(root), int(mode), _ptr(parents), _ptr(distances),
                                        C.byref(info), _stream(stream)), "ogb_bfs")
        return info_dict(info)

    def msbfs(self, roots, depths, stream=None) -> dict:
        """Up to 64 searches at once; depths is a device uint16/int16 tensor
        of V * 64 entries (row v = v's depth in each lane, 0xFFFF unreached)."""
        arr = (u32 * len(roots))(*[int(r) for r in roots])
        info = MsBfsInfo()
        self.lib.check(self.lib.ogb_msbfs(self.handle, arr, len(roots), _ptr(depths), C.byref(info), _stream(stream)),
                       "ogb_msbfs")
        return info_dict(info)

    def ppr(self, seeds, ranks=None, max_iterations: int = 20, epsilon: float = 0.0, stream=None) -> dict:
        """Personalized PageRank for up to 32 one-hot seeds; ranks (device
        float32, V * 32) receives row v = v's rank in each seed's vector."""
        arr = (u32 * len(seeds))(*[int(x) for x in seeds])
        info = PprBatchInfo()
        self.lib.check(self.lib.ogb_ppr(self.handle, arr, len(seeds), int(max_iterations), float(epsilon),
                                        _ptr(ranks), C.byref(info), _stream(stream)), "ogb_ppr")
        d = info_dict(info)
        d["err_last"] = list(info.err_last)[:len(seeds)]
        return d

    def bfs_features(self, max_levels: int = 16384) -> np.ndarray:
        """The learned switch's inputs before every step of the last bfs."""
        out = np.zeros((max_levels, 8), np.float32)
        n = u32()
        self.lib.check(self.lib.ogb_bfs_features(self.handle, out.ctypes.data, max_levels, C.byref(n)),
                       "ogb_bfs_features")
        return out[:n.value].copy()

    def pagerank_warm_start(self, params, init, hidden: int = 32, stream=None) -> None:
        p = np.ascontiguousarray(np.asarray(params, np.float32))
        self.lib.check(self.lib.ogb_pagerank_warm_start(self.handle, hidden, p.ctypes.data, _ptr(init), _stream(stream)),
                       "ogb_pagerank_warm_start")

    def bfs_trace(self, max_levels: int = 16384) -> list[dict]:
        arr = (BfsLevel * max_levels)()
        n = u32()
        self.lib.check(self.lib.ogb_bfs_trace(self.handle, arr, max_levels, C.byref(n)), "ogb_bfs_trace")
        return [info_dict(arr[i]) for i in range(n.value)]

    def pagerank(self, ranks, mode: int = 0, max_iterations: int = 20, epsilon: float = 1e-4, init=None,
                 stream=None) -> dict:
        info = PrInfo()
        self.lib.check(self.lib.ogb_pagerank(self.handle, int(mode), int(max_iterations), float(epsilon),
                                             _ptr(ranks), _ptr(init), C.byref(info), _stream(stream)), "ogb_pagerank")
        return info_dict(info)

    def spmv(self, x, y, mode: int = 0, iterations: int = 20, stream=None) -> dict:
        """SPMV (mode 0 pull, 1 push): x receives the input vector, y the
        output accumulated over `iterations` passes (device float32, V)."""
        info = SpmvInfo()
        self.lib.check(self.lib.ogb_spmv(self.handle, int(mode), int(iterations), _ptr(x), _ptr(y), C.byref(info),
                                         _stream(stream)), "ogb_spmv")
        return info_dict(info)

    def pagerank_history(self, max_entries: int = 1024) -> tuple[np.ndarray, np.ndarray]:
        err = (C.c_double * max_entries)()
        act = (u32 * max_entries)()
        n = u32()
        self.lib.check(self.lib.ogb_pagerank_history(self.handle, err, act, max_entries, C.byref(n)), "history")
        return np.array(err[:n.value]), np.array(act[:n.value], dtype=np.uint32)


# -------------------------------------------------------------- generators --

def sort_by_rank(lib, ranks, labels, stream=None) -> None:
    """radixSortEdgesByPageRank on device tensors: labels (int32/uint32, n)
    sorted in place by the fixed-point key of ranks (float32, n)."""
    lib.check(lib.ogb_sort_by_rank(_ptr(ranks), _ptr(labels), int(labels.numel()), _stream(stream)),
              "ogb_sort_by_rank")


def generate_rmat(scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19, permute=True,
                  weighted=False, lib: Library | None = None):
    """Graph500 RMAT edge list on the host (numpy uint32 src, dst[, float32 w])."""
    lib = lib or load(False)
    E = (1 << scale) * edge_factor
    src = np.empty(E, np.uint32)
    dst = np.empty(E, np.uint32)
    w = np.empty(E, np.float32) if weighted else None
    lib.check(lib.ogb_generate_rmat(scale, edge_factor, seed, a, b, c, 1 if permute else 0, src.ctypes.data,
                                    dst.ctypes.data, w.ctypes.data if w is not None else None), "generate_rmat")
    return src, dst, w


def generate_uniform(num_vertices: int, num_edges: int, seed: int, weighted=False, lib: Library | None = None):
    lib = lib or load(False)
    src = np.empty(num_edges, np.uint32)
    dst = np.empty(num_edges, np.uint32)
    w = np.empty(num_edges, np.float32) if weighted else None
    lib.check(lib.ogb_generate_uniform(num_vertices, num_edges, seed, src.ctypes.data, dst.ctypes.data,
                                       w.ctypes.data if w is not None else None), "generate_uniform")
    return src, dst, w


def generate_grid(side: int, p: float, seed: int, weighted=False, lib: Library | None = None):
    lib = lib or load(False)
    n = C.c_uint64()
    lib.check(lib.ogb_generate_grid(side, p, seed, None, None, None, C.byref(n)), "generate_grid")
    src = np.empty(n.value, np.uint32)
    dst = np.empty(n.value, np.uint32)
    w = np.empty(n.value, np.float32) if weighted else None
    lib.check(lib.ogb_generate_grid(side, p, seed, src.ctypes.data, dst.ctypes.data,
                                    w.ctypes.data if w is not None else None, C.byref(n)), "generate_grid")
    return src, dst, w


def write_edge_file(path: str, src, dst, w=None, lib: Library | None = None) -> None:
    """Reference .bin (8-byte records) or .wbin (12-byte records with w)."""
    lib = lib or load(False)
    lib.check(lib.ogb_write_edge_file(path.encode(), src.ctypes.data, dst.ctypes.data,
                                      w.ctypes.data if w is not None else None, len(src)), "write_edge_file")
