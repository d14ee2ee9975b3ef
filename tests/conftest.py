"""Shared fixtures: the product library (both layouts), the oracle, the
reference's CPU build, and seeded synthetic graphs."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

os.environ.setdefault("OGB200_QUIET", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")
    config.addinivalue_line("markers", "slow: full-size checks (scale 22)")


def _cuda_ok() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_ok():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def og():
    import opengraph_b200 as og
    return og


@pytest.fixture(scope="session")
def lib(og):
    lib = og.load(False)
    lib.quiet(True)
    return lib


@pytest.fixture(scope="session")
def libw(og):
    lib = og.load(True)
    lib.quiet(True)
    return lib


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


def _ref(weighted):
    from oracle.oracle import Reference
    if not Reference.available(weighted):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    return Reference(weighted)


@pytest.fixture(scope="session")
def ref():
    return _ref(False)


@pytest.fixture(scope="session")
def refw():
    return _ref(True)


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    torch.cuda.init()
    return torch


_GRAPH_CACHE: dict = {}


def graph_edges(kind: str, **kw):
    """Seeded synthetic edge lists (cached): rmat, uniform, grid, and small
    hand-made edge cases."""
    import opengraph_b200 as og
    key = (kind, tuple(sorted(kw.items())))
    if key in _GRAPH_CACHE:
        return _GRAPH_CACHE[key]
    weighted = kw.get("weighted", False)
    if kind == "rmat":
        s, d, w = og.generate_rmat(kw["scale"], kw.get("ef", 16), kw.get("seed", 0), weighted=weighted)
    elif kind == "uniform":
        s, d, w = og.generate_uniform(kw["n"], kw["m"], kw.get("seed", 0), weighted=weighted)
    elif kind == "grid":
        s, d, w = og.generate_grid(kw["side"], kw.get("p", 1e-2), kw.get("seed", 0), weighted=weighted)
    elif kind == "star":  # hub with many duplicates and self loops
        n = kw.get("n", 5000)
        rng = np.random.default_rng(kw.get("seed", 0))
        s = np.concatenate([np.zeros(n, np.uint32), rng.integers(0, 64, n).astype(np.uint32)])
        d = np.concatenate([rng.integers(0, 64, n).astype(np.uint32), np.zeros(n, np.uint32)])
        w = rng.uniform(1, 256, len(s)).astype(np.float32) if weighted else None
    elif kind == "chain":  # long path: many levels
        n = kw.get("n", 3000)
        s = np.arange(n - 1, dtype=np.uint32)
        d = s + 1
        w = np.ones(len(s), np.float32) if weighted else None
    else:
        raise KeyError(kind)
    V = int(max(s.max(initial=0), d.max(initial=0))) + 1 if len(s) else 1
    out = (s, d, w, V)
    _GRAPH_CACHE[key] = out
    return out


@pytest.fixture(scope="session")
def graphs():
    return graph_edges
