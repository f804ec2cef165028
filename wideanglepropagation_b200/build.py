"""Build libwap.so in-tree for sm_100a.

``python -m wideanglepropagation_b200.build`` compiles every CUDA source under
``csrc/`` into ``wideanglepropagation_b200/libwap.so`` (nvcc, -gencode
arch=compute_100a,code=sm_100a, -lineinfo).  Sources compile to objects in
parallel under ``_build/`` (one nvcc per source) and are linked into the
library; a source recompiles when it, or any header, is newer than its object.
Rebuilds only when a source is newer than the library unless ``force``.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
DEPS = SRC + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
    sorted(glob.glob(os.path.join(HERE, "csrc", "*.h"))) + [os.path.join(ROOT, "include", "wap.h")]
HEADERS = [p for p in DEPS if not p.endswith(".cu")]
OUT = os.path.join(HERE, "libwap.so")
OBJDIR = os.path.join(ROOT, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in DEPS)


def _obj(src: str) -> str:
    return os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")


def _stale(src: str, newest_header: float) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return os.path.getmtime(src) > t or newest_header > t


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    os.makedirs(OBJDIR, exist_ok=True)
    newest_header = max(os.path.getmtime(p) for p in HEADERS)
    todo = [s for s in SRC if force or _stale(s, newest_header)]
    flags = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC"]
    if verbose:
        flags += ["-Xptxas", "-v"]

    def compile_one(src: str):
        tmp = _obj(src) + ".tmp"
        r = subprocess.run([nvcc(), *flags, "-c", src, "-o", tmp], capture_output=True, text=True)
        if r.returncode == 0:
            os.replace(tmp, _obj(src))
        return src, r

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, todo))
    failed = [(src, r) for src, r in results if r.returncode != 0]
    for src, r in results:
        if verbose or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(os.path.basename(s) for s, _ in failed))
    tmp = OUT + ".tmp"
    r = subprocess.run([nvcc(), *ARCH, "-shared", "-o", tmp, *[_obj(s) for s in SRC]],
                       capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libwap.so")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
