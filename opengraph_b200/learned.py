"""The learned parts beside the plain path: a direction-switch policy for BFS
and a warm-start vector for PageRank, trained on the GPU by the library's
own MLP kernels (ogb_mlp_train) on traces of the plain GPU runs, and used by
hand-written inference kernels (bf16 weights, fp32 accumulation).

  python -m opengraph_b200.learned train [dir]        # writes opengraph_b200/weights/*.f32 (or dir)
  python -m opengraph_b200.learned collect s.npz      # only the training traces
  python -m opengraph_b200.learned fit s.npz [dir]    # only the fit, from saved traces
  python -m opengraph_b200.learned evaluate           # learned vs plain on held-out graphs

Direction switch (8 -> 64 -> 64 -> 1 network plus a linear prior; a step
runs bottom-up when prior(x) + clamp(network(x), -B, B) > 0).  Every BFS
level has the same frontier whatever the directions chosen before it (the
search is level-synchronous), so a push-only and a pull-only search from one
root give, level by level, the device time of a top-down and of a bottom-up
step on the same frontier.  Training samples: the switch inputs the kernel
records before each level (ogb_bfs_features), with target
y = log2(top-down ms / bottom-up ms) (clipped to +-8).  The prior is a
least-squares fit of y on L(frontier out-edges) (the reference rule's mf,
BFS.c:520-560), L(bottom-up candidates) (the list a bottom-up step would
walk: the graph's vertices with in-edges before the first bottom-up step,
the unvisited list after it, all V in the dense probe) and the list flag: a power-law model of the two steps' costs, top-down work growing
with the frontier's edges and bottom-up work with its candidates.  The
network is fitted (squared error) to the remaining residual, clipped to +-B,
so far from the training states it can move the decision by at most B and
the prior decides.  (A prior on more counts fits the training graphs
slightly better but extrapolates worse: with L(unexplored out-edges) and
L(V) in it, the tail of a 4096 x 4096 grid search looks like an RMAT tail,
where bottom-up wins, while a bottom-up step there walks 16M vertices.)
The plain alpha/beta rule stays the default (mode 2); mode 3 uses the
policy; depths are identical by construction.

PageRank warm start (2 -> 32 -> 32 -> 1): inputs log2(1 + in-degree),
log2(1 + out-degree); target log2 of the vertex's unnormalized rank after
the plain pull run (100 iterations).  The start vector 2^prediction replaces
the uniform 1 - 0.85 (pageRank.c:68); the iteration and its stop rule are
unchanged, so the run converges to the same ranks (within the tolerance).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights")
# (file, inputs, hidden units, extra floats after the network)
SWITCH = ("switch_mlp.f32", 8, 64, 10)   # + prior coefficients[8], prior bias, correction bound
PR_START = ("pr_start_mlp.f32", 2, 32, 0)
SWITCH_BOUND = 2.0                        # B: the network moves log2(td / bu) by at most 2
PRIOR_INPUTS = (1, 3, 7)                  # L(frontier out-edges), L(bottom-up candidates), list flag


def weights_path(spec) -> str:
    return os.path.join(WEIGHTS, spec[0])


def load_weights(lib, spec) -> np.ndarray | None:
    """The committed fp32 parameters of a network, or None when absent."""
    import opengraph_b200 as og
    p = weights_path(spec)
    if not os.path.exists(p):
        return None
    w = np.fromfile(p, dtype=np.float32)
    want = og.mlp_nparams(lib, spec[1], spec[2]) + spec[3]
    if len(w) != want:
        raise ValueError(f"{p}: {len(w)} parameters, expected {want}")
    return w


def _device_graph(lib, s, d, V):
    import torch
    g = lib.device_graph()
    g.build(torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda(), V, 0)
    return g


def _roots(g, n, seed):
    outdeg = g.view(False).out_degree.cpu().numpy().view(np.uint32)
    rng = np.random.default_rng(seed)
    cand = np.nonzero(outdeg > 0)[0]
    return [int(x) for x in rng.choice(cand, size=min(n, len(cand)), replace=False)]


def switch_samples(lib, g, V, roots):
    """(features, log2(td ms / bu ms)) per level: positive when the bottom-up
    step on that level's frontier was faster than the top-down step.  Two
    samples per level: a bottom-up step over all vertices (inputs of the
    push-only search, candidates = V; timed by the dense pull probe, mode 4)
    and one over the unvisited list (inputs of the pull-only search, whose
    steps after its first walk the list)."""
    import torch
    par = torch.empty(V, dtype=torch.int32, device="cuda")
    dist = torch.empty(V, dtype=torch.int32, device="cuda")
    X, Y = [], []

    def ratio(a, b):
        return np.clip(np.log2(np.maximum(np.asarray(a), 1e-4) / np.maximum(np.asarray(b), 1e-4)), -8, 8)

    for r in roots:
        g.bfs(r, par, dist, mode=1)            # push only
        td = [L["ms"] for L in g.bfs_trace()]
        feat_push = g.bfs_features()
        g.bfs(r, par, dist, mode=4)            # pull, every step over all vertices
        dense = [L["ms"] for L in g.bfs_trace()]
        g.bfs(r, par, dist, mode=0)            # pull, unvisited list after the first step
        lst = [L["ms"] for L in g.bfs_trace()]
        feat_pull = g.bfs_features()
        n = min(len(td), len(dense), len(feat_push))
        X.append(feat_push[:n])
        Y.append(ratio(td[:n], dense[:n]).astype(np.float32))
        m = min(len(td), len(lst), len(feat_pull))
        if m > 1:
            X.append(feat_pull[1:m])
            Y.append(ratio(td[1:m], lst[1:m]).astype(np.float32))
    return np.concatenate(X), np.concatenate(Y)


def pr_samples(lib, g, V, n_samples, seed):
    """(features, target) for a random subset of vertices."""
    import torch
    ranks = torch.empty(V, dtype=torch.float32, device="cuda")
    g.pagerank(ranks, mode=0, max_iterations=100, epsilon=0.0)
    r = ranks.cpu().numpy().astype(np.float64) * V       # unnormalized
    indeg = g.view(True).out_degree.cpu().numpy().view(np.uint32).astype(np.float64)
    outdeg = g.view(False).out_degree.cpu().numpy().view(np.uint32).astype(np.float64)
    rng = np.random.default_rng(seed)
    idx = rng.choice(V, size=min(n_samples, V), replace=False)
    X = np.stack([np.log2(1 + indeg[idx]), np.log2(1 + outdeg[idx])], axis=1).astype(np.float32)
    Y = np.log2(np.maximum(r[idx], 1e-30)).astype(np.float32)
    return X, Y


def collect(scales=(18, 19, 20, 21, 22), seeds=tuple(range(32)), roots_per_graph=4, pr_per_graph=25_000, log=print):
    """Training samples from plain GPU runs on RMAT graphs (edge factor 16,
    generator seeds 100 + seed): switch (X, y) from every root's levels and
    warm-start (X, y) from a vertex subset of every graph."""
    import opengraph_b200 as og
    lib = og.load(False)
    lib.quiet(True)
    Xs, Ys, Xp, Yp = [], [], [], []
    for sc in scales:
        for sd in seeds:
            s, d, _ = og.generate_rmat(sc, 16, 100 + sd)
            V = 1 << sc
            g = _device_graph(lib, s, d, V)
            x, y = switch_samples(lib, g, V, _roots(g, roots_per_graph, sd))
            Xs.append(x)
            Ys.append(y)
            x, y = pr_samples(lib, g, V, pr_per_graph, sd)
            Xp.append(x)
            Yp.append(y)
            g.close()
        log(f"traces: RMAT-{sc}, {len(seeds)} seeds")
    return {"switch_X": np.concatenate(Xs), "switch_y": np.concatenate(Ys),
            "pr_X": np.concatenate(Xp), "pr_y": np.concatenate(Yp)}


def fit_prior(X, y):
    """Least squares y ~ sum_i a_i * X[:, i] (i in PRIOR_INPUTS) + b; returns
    the 10-float tail (coefficients[8], bias, bound)."""
    cols = list(PRIOR_INPUTS)
    A = np.concatenate([X[:, cols].astype(np.float64), np.ones((len(X), 1))], axis=1)
    coef, *_ = np.linalg.lstsq(A, y.astype(np.float64), rcond=None)
    tail = np.zeros(10, np.float32)
    tail[cols] = coef[:-1]
    tail[8] = coef[-1]
    tail[9] = SWITCH_BOUND
    return tail


def prior_of(tail, X):
    return X.astype(np.float64) @ tail[:8].astype(np.float64) + float(tail[8])


def fit(samples, out=WEIGHTS, log=print):
    """Train the networks whose samples are given (switch_X/switch_y,
    pr_X/pr_y) on the GPU (ogb_mlp_train) and write their files."""
    import torch

    import opengraph_b200 as og
    lib = og.load(False)
    os.makedirs(out, exist_ok=True)
    res = {}
    jobs = []
    if "switch_X" in samples:
        Xs, ys = samples["switch_X"], samples["switch_y"]
        tail = fit_prior(Xs, ys)
        resid = np.clip(ys - prior_of(tail, Xs), -SWITCH_BOUND, SWITCH_BOUND).astype(np.float32)
        jobs.append(("switch", (Xs, resid), SWITCH, 0, 600, 128, 1e-3))
    if "pr_X" in samples:
        jobs.append(("pr_start", (samples["pr_X"], samples["pr_y"]), PR_START, 0, 30, 4096, 2e-3))
    for name, (X, Y), spec, loss, epochs, batch, lr in jobs:
        tx = torch.from_numpy(np.ascontiguousarray(X)).cuda()
        ty = torch.from_numpy(np.ascontiguousarray(Y)).cuda()
        p0 = og.mlp_init(lib, spec[1], spec[2], seed=7)
        p, hist = og.mlp_train(lib, spec[1], spec[2], loss, tx, ty, p0, epochs=epochs, batch=batch, lr=lr, seed=11)
        blob = np.concatenate([p.astype(np.float32), tail]) if name == "switch" else p.astype(np.float32)
        blob.tofile(os.path.join(out, spec[0]))
        res[name] = {"samples": int(len(Y)), "loss_first": float(hist[0]), "loss_last": float(hist[-1])}
        if name == "switch":
            res[name]["bottom_up_faster_fraction"] = float((ys > 0).mean())
            res[name]["prior"] = {"coefficients": [float(x) for x in tail[:8]], "bias": float(tail[8]),
                                  "residual_rms": float(np.sqrt(np.mean(resid.astype(np.float64) ** 2)))}
        log(f"{name}: {res[name]}")
    return res


def train(out=WEIGHTS, log=print, **kw):
    return fit(collect(log=log, **kw), out=out, log=log)


def evaluate(log=print, grid_roots=8):
    """Learned vs plain on held-out graphs: RMAT-24 (a seed never used in
    training; 32 random roots) and a 4096 x 4096 grid with random shortcuts
    (p = 1e-4; 8 roots, about 0.15 s per search)."""
    import torch

    import opengraph_b200 as og
    lib = og.load(False)
    lib.quiet(True)
    sw = load_weights(lib, SWITCH)
    pw = load_weights(lib, PR_START)
    if sw is None or pw is None:
        raise SystemExit("no trained weights: run `python -m opengraph_b200.learned train` first")
    lib.check(lib.ogb_bfs_set_policy(sw.ctypes.data), "ogb_bfs_set_policy")
    out = {}
    graphs = [("rmat24_seed900", lambda: og.generate_rmat(24, 16, 900)[:2], 1 << 24, 32),
              ("grid4096_p1e-4", lambda: og.generate_grid(4096, 1e-4, 901)[:2], 4096 * 4096, grid_roots)]
    for name, gen, V, nroots in graphs:
        s, d = gen()
        g = _device_graph(lib, s, d, V)
        par = torch.empty(V, dtype=torch.int32, device="cuda")
        dist = torch.empty(V, dtype=torch.int32, device="cuda")
        roots = _roots(g, nroots, 77)
        tot = {"plain": [0.0, 0.0], "learned": [0.0, 0.0]}
        same = True
        plain_depths = torch.empty_like(dist)
        for r in roots:   # both switches per root, depths compared on the device
            for mode, tag in ((2, "plain"), (3, "learned")):
                g.bfs(r, par, dist, mode=mode)
                info = g.bfs(r, par, dist, mode=mode)
                tot[tag][0] += info["ms"]
                tot[tag][1] += info["reached_out_edges"]
                if tag == "plain":
                    plain_depths.copy_(dist)
                else:
                    same = same and bool(torch.equal(dist, plain_depths))
        bfs = {t: {"gteps": round(e / ms / 1e6, 4), "ms_per_search": round(ms / len(roots), 4)}
               for t, (ms, e) in tot.items()}
        bfs["roots"] = len(roots)
        bfs["depths_identical"] = bool(same)
        # PageRank: iterations until the L1 change of normalized ranks < 1e-6
        ranks = torch.empty(V, dtype=torch.float32, device="cuda")
        init = torch.empty(V, dtype=torch.float32, device="cuda")
        pr = {}
        for tag in ("plain", "learned"):
            if tag == "learned":
                g.pagerank_warm_start(pw, init, hidden=PR_START[2])
                start = init
            else:
                start = None
            info = g.pagerank(ranks, mode=0, max_iterations=200, epsilon=0.0, init=start)
            errs, _ = g.pagerank_history()
            hit = next((i for i, e in enumerate(errs) if e < 1e-6), None)
            it_ms = info["ms"] / 200
            pr[tag] = {"iterations_to_1e-6": (hit + 1) if hit is not None else None,
                       "ms_to_1e-6": round(it_ms * (hit + 1), 3) if hit is not None else None,
                       "ranks": ranks.cpu().numpy().astype(np.float64)}
        l1 = float(np.abs(pr["plain"].pop("ranks") - pr["learned"].pop("ranks")).sum())
        pr["final_l1_between"] = l1
        out[name] = {"bfs": bfs, "pagerank": pr}
        log(f"{name}: {json.dumps(out[name])}")
        g.close()
    lib.ogb_bfs_set_policy(None)
    return out


if __name__ == "__main__":
    cmd = sys.argv[1] if len(sys.argv) > 1 else "evaluate"
    if cmd == "train":
        print(json.dumps(train(out=sys.argv[2] if len(sys.argv) > 2 else WEIGHTS)))
    elif cmd == "collect":        # collect samples.npz: the traces alone
        np.savez_compressed(sys.argv[2], **collect())
    elif cmd == "fit":            # fit samples.npz [dir]: the networks from saved traces
        z = np.load(sys.argv[2])
        print(json.dumps(fit({k: z[k] for k in z.files}, out=sys.argv[3] if len(sys.argv) > 3 else WEIGHTS)))
    else:
        print(json.dumps(evaluate()))
