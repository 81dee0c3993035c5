"""Build the sm_100a shared library ``bosss_b200/libbosss_b200.so`` in-tree.

Every CUDA translation unit is compiled by nvcc for ``sm_100a`` only
(``-gencode arch=compute_100a,code=sm_100a``); the objects are linked into one
shared library exporting the C-ABI of ``include/bosss_b200.h``. Translation units
are compiled in parallel and skipped when their object is newer than the unit and every
local header it includes.

Usage: ``python -m bosss_b200.build [--force] [-j N]``
"""
import argparse
import glob
import os
import re
import shutil
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbosss_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"),
    # no --split-compile: it partitions a unit's kernels for parallel optimisation and
    # measurably slowed the Euler VJP kernel (0.59 -> 0.68 ms at 32^3, k=3)
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src, seen=None):
    """Local headers a translation unit includes, transitively (quoted includes only)."""
    seen = set() if seen is None else seen
    try:
        with open(src) as f:
            text = f.read()
    except OSError:
        return seen
    for inc in _INCLUDE.findall(text):
        path = os.path.normpath(os.path.join(os.path.dirname(src), inc))
        if path not in seen and os.path.exists(path):
            seen.add(path)
            _deps(path, seen)
    return seen


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in inputs)


def build(force=False, jobs=None, verbose=False):
    """Compile every CUDA translation unit and link the shared library; returns its path."""
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()
    objs, todo = [], []
    for src in _sources():
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + sorted(_deps(src))):
            todo.append((src, obj))

    def compile_one(item):
        src, obj = item
        cmd = [cc] + NVCC_FLAGS + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        t0 = time.time()
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
        # the object reflects the sources as they were when the compile started: a header
        # edited during a long compile leaves it stale
        os.utime(obj, (t0, t0))
        return src

    if todo:
        jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
        # biggest translation units first
        todo.sort(key=lambda it: -os.path.getsize(it[0]))
        with ThreadPoolExecutor(max_workers=jobs) as ex:
            for src in ex.map(compile_one, todo):
                if verbose:
                    print("compiled", os.path.basename(src), flush=True)
    if force or todo or _stale(LIB, objs):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.j, verbose=a.v))


if __name__ == "__main__":
    sys.exit(main())
