"""Build libdgfock.so (the CUDA kernels and the C ABI) for sm_100a, in-tree.

Each ``csrc/*.cu`` file, and one generated unit per quartet-class pair of
the Fock and gradient kernel tables, is compiled to an object in parallel,
then linked into ``dalton_b200/libdgfock.so``.  Objects are rebuilt only when
a source or header is newer.
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


NUM_PAIR_CLASS = 10  # (la >= lb) shell-pair classes up to f
NUM_GRAD_CLASS = 6   # the gradient covers s, p and d


def _class_l(x):
    la = 0 if x == 0 else 1 if x <= 2 else 2 if x <= 5 else 3
    return la + (x - la * (la + 1) // 2)


def _generated_units():
    """One translation unit per class pair of the Fock and gradient kernel
    tables (their templates live in headers), written to the build folder
    only when the content changes; heaviest classes first."""
    gen = os.path.join(BUILD, "gen")
    os.makedirs(gen, exist_ok=True)
    units = []
    for kind, header, macro, n, parts in (("jk", None, None, NUM_PAIR_CLASS, 3),
                                          ("grad", "dgf_grad_kernel.cuh", "DGF_GRAD_CLASS", NUM_GRAD_CLASS, 0)):
        for x in range(n):
            for y in range(x + 1):
                for part in (range(parts) if parts else [None]):
                    if part is None:
                        path = os.path.join(gen, f"dgf_{kind}_{x}_{y}.cu")
                        text = f'#include "{header}"\n\n{macro}({x}, {y})\n'
                    elif part == 0:  # cooperative, warp-team and warp-per-quartet kernels
                        path = os.path.join(gen, f"dgf_{kind}_{x}_{y}_0.cu")
                        text = f'#include "dgf_jk_inst_team.cuh"\n\nDGF_JK_TEAM_CLASS({x}, {y})\n'
                    else:  # thread kernels, FP64 (1) or FP32 (2)
                        path = os.path.join(gen, f"dgf_{kind}_{x}_{y}_{part}.cu")
                        text = f'#include "dgf_jk_inst_thread.cuh"\n\nDGF_JK_THREAD_CLASS({x}, {y}, {part})\n'
                    if not os.path.exists(path) or open(path).read() != text:
                        with open(path, "w") as f:
                            f.write(text)
                    units.append((_class_l(x) + _class_l(y), path))
    # drop objects of units that are no longer generated (an earlier layout)
    keep = {os.path.basename(p).replace(".cu", ".o") for _, p in units}
    for o in glob.glob(os.path.join(BUILD, "dgf_jk_*.o")):
        if os.path.basename(o) not in keep:
            os.remove(o)
    for g in glob.glob(os.path.join(gen, "dgf_jk_*.cu")):
        if os.path.basename(g).replace(".cu", ".o") not in keep:
            os.remove(g)
    return [p for _, p in sorted(units, key=lambda u: -u[0])]


def build(verbose: bool = False, extra=None, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = _generated_units() + sorted(glob.glob(os.path.join(CSRC, "*.cu")))
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
