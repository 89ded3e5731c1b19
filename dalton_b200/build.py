"""Build libdgfock.so (the CUDA kernels and the C ABI) for sm_100a, in-tree.

Each ``csrc/*.cu`` file is compiled to an object in parallel, then linked
into ``dalton_b200/libdgfock.so``.  Objects are rebuilt only when a source or
header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdgfock.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-ccbin", "g++", "-I", INCLUDE, "-I", CSRC]


def _deps(path, seen=None):
    """Local headers a source includes, recursively (#include "...")."""
    seen = set() if seen is None else seen
    with open(path) as f:
        for line in f:
            m = re.match(r'\s*#\s*include\s+"([^"]+)"', line)
            if not m:
                continue
            for base in (os.path.dirname(path), CSRC, INCLUDE):
                cand = os.path.normpath(os.path.join(base, m.group(1)))
                if os.path.exists(cand):
                    if cand not in seen:
                        seen.add(cand)
                        _deps(cand, seen)
                    break
    return seen


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    if not _stale(obj, [src] + sorted(_deps(src))):
        return obj, ""
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False, extra=None, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    extra = list(extra or [])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        res = list(ex.map(lambda s: _compile(s, extra), srcs))
    objs = [o for o, _ in res]
    if verbose:
        for _, err in res:
            if err.strip():
                print(err)
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build(verbose=v, extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None))
