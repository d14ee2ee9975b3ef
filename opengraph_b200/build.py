"""Build libogb200.so (WEIGHTED=0 layout) and libogb200_w.so (WEIGHTED=1) in-tree.

Every CUDA source is compiled for sm_100a only; cudart is linked statically so
the libraries load without a CUDA library path.  Usage:
    python -m opengraph_b200.build [--force] [-v]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")

CUDA_SOURCES = ["graph.cu", "sort.cu", "scan.cu", "bfs.cu", "bfs_range.cu", "partition.cu", "pagerank.cu", "compact.cu",
                "noalloc.cu", "batch.cu", "mlp.cu", "dd.cu"]
LAYOUT_SOURCES = ["abi.cu"]  # compiled once per struct layout
CXX_SOURCES = ["generate.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3,-fopenmp", "--expt-relaxed-constexpr",
              "-I", INCLUDE, "-I", CSRC] + ARCH

LIBS = {"libogb200.so": 0, "libogb200_w.so": 1}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:4]) + " ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def _sources_present() -> list[str]:
    return [s for s in CUDA_SOURCES if os.path.exists(os.path.join(CSRC, s))]


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> list[str]:
    os.makedirs(BUILD, exist_ok=True)
    nv = nvcc()
    hdrs = _headers()
    flags = NVCC_FLAGS + (extra_flags or [])
    jobs = []  # (obj, cmd, deps)
    for src in _sources_present():
        obj = os.path.join(BUILD, src + ".o")
        deps = [os.path.join(CSRC, src)] + hdrs
        jobs.append((obj, [nv, *flags, "-c", os.path.join(CSRC, src), "-o", obj], deps))
    for src in CXX_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        deps = [os.path.join(CSRC, src)] + hdrs
        jobs.append((obj, [nv, *flags, "-x", "cu", "-c", os.path.join(CSRC, src), "-o", obj], deps))
    for lib, w in LIBS.items():
        for src in LAYOUT_SOURCES:
            obj = os.path.join(BUILD, f"{src}.w{w}.o")
            deps = [os.path.join(CSRC, src)] + hdrs
            jobs.append((obj, [nv, *flags, f"-DOGB200_WEIGHTED={w}", "-c", os.path.join(CSRC, src), "-o", obj], deps))
    todo = [(o, c) for o, c, d in jobs if force or not _newer(o, d)]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(lambda oc: _run(oc[1], verbose), todo))
    common = [os.path.join(BUILD, s + ".o") for s in _sources_present() + CXX_SOURCES]
    out = []
    for lib, w in LIBS.items():
        objs = common + [os.path.join(BUILD, f"{s}.w{w}.o") for s in LAYOUT_SOURCES]
        target = os.path.join(HERE, lib)
        if force or not _newer(target, objs):
            _run([nv, *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC",
                  "-Xlinker", "-Bsymbolic-functions", "-o", target, *objs, "-lgomp", "-lpthread"], verbose)
        out.append(target)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    for p in build(force=a.force, verbose=a.verbose):
        print(p)


if __name__ == "__main__":
    main()
