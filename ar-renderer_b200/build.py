"""Builds the native libraries of the package in-tree.

* ``libprender_gpu.so`` -- the CUDA module (csrc/*.cu) for sm_100a, exporting the C ABI declared
  in include/prgpu_api.h.
* ``libprender_host.so`` -- the C++ host library (host/*.cpp): BVH and light-BVH builders and
  spectral tabulation, exporting include/prhost_api.h.

Run ``python ar-renderer_b200/build.py`` (or ``__graft_entry__.build()``). Objects are rebuilt only
when a source or header is newer than the library.
"""

from __future__ import annotations

import os
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")

GPU_LIB = os.path.join(PKG, "libprender_gpu.so")
HOST_LIB = os.path.join(PKG, "libprender_host.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I", INCLUDE,
]
# Shading and the verification kernels round every product before it is added (no FMA
# contraction), as the reference's ISO C++ build does, so BxDF / phase / medium values agree
# with it to a few ulps even where the formulas cancel.
PER_FILE_FLAGS = {"render.cu": ["--fmad=false"], "batch.cu": ["--fmad=false"], "funcs.cu": ["--fmad=false"]}
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off", "-I", INCLUDE,
             "-pthread"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _newest(paths) -> float:
    return max((os.path.getmtime(p) for p in paths if os.path.exists(p)), default=0.0)


def _sources(d: str, exts) -> list[str]:
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts))


def _local_includes(path: str, seen: set | None = None) -> set:
    """The file and every header it includes with quotes, transitively (resolved beside the
    including file, then in include/)."""
    seen = set() if seen is None else seen
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path, errors="replace") as f:
        for line in f:
            line = line.strip()
            if line.startswith("#include \""):
                name = line.split('"')[1]
                for base in (os.path.dirname(path), INCLUDE):
                    cand = os.path.normpath(os.path.join(base, name))
                    if os.path.exists(cand):
                        _local_includes(cand, seen)
                        break
    return seen


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build_gpu(force: bool = False, verbose: bool = False) -> str:
    srcs = _sources(CSRC, (".cu",))
    deps = srcs + _sources(CSRC, (".cuh", ".h")) + _sources(INCLUDE, (".h",))
    if not force and os.path.exists(GPU_LIB) and os.path.getmtime(GPU_LIB) >= _newest(deps):
        return GPU_LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    objs = []

    def compile_one(src: str) -> str:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        # An object is current when it is newer than its source and the headers that source reaches.
        if not force and not verbose and os.path.exists(obj) and \
                os.path.getmtime(obj) >= _newest(_local_includes(src)) and os.path.getmtime(obj) >= os.path.getmtime(__file__):
            return obj
        cmd = [nvcc, *NVCC_FLAGS, *PER_FILE_FLAGS.get(os.path.basename(src), []), "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        started = time.time()
        _run(cmd)
        # Date the object at the start of its compile, so a source edited meanwhile is newer.
        os.utime(obj, (started, started))
        return obj

    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    # Static CUDA runtime: the library needs no LD_LIBRARY_PATH and shares the primary context.
    _run([nvcc, "-shared", "-cudart", "static", "-o", GPU_LIB, *objs, "-Xlinker", "--exclude-libs,ALL"])
    return GPU_LIB


def build_host(force: bool = False) -> str:
    srcs = _sources(HOST, (".cpp",))
    if not srcs:
        return ""
    deps = srcs + _sources(HOST, (".h", ".hpp")) + _sources(INCLUDE, (".h",))
    if not force and os.path.exists(HOST_LIB) and os.path.getmtime(HOST_LIB) >= _newest(deps):
        return HOST_LIB
    cxx = os.environ.get("CXX", "g++")
    # Symbols of statically linked runtime libraries stay private to the library.
    _run([cxx, *CXX_FLAGS, "-shared", "-o", HOST_LIB, *srcs, "-Wl,--exclude-libs,ALL"])
    return HOST_LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_gpu(force=force, verbose=verbose)
    build_host(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", GPU_LIB, HOST_LIB)
