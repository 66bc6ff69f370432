"""Builds libgolb200.so (the engine's C ABI) in place for sm_100a.

    python stencil-optimalizations_b200/build.py [--force] [--verbose]

nvcc compiles the CUDA kernels, the engine and the host packing code (one
object per source, in parallel, under _build/) and links them into one
shared library next to this file; rebuilt only when a source is newer.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libgolb200.so")
INCLUDE = os.path.join(ROOT, "include")
OBJ_DIR = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC,-O3",
    "-shared",
]


def sources() -> list[str]:
    srcs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    srcs += sorted(glob.glob(os.path.join(HERE, "csrc", "*.cpp")))
    return srcs


def deps() -> list[str]:
    return sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
        sorted(glob.glob(os.path.join(HERE, "csrc", "*.h"))) + \
        sorted(glob.glob(os.path.join(INCLUDE, "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _compile(src: str, obj: str, verbose: bool) -> None:
    cmd = [nvcc(), *[f for f in NVCC_FLAGS if f != "-shared"], f"-I{INCLUDE}", "-c", src, "-o", obj]
    if verbose:
        cmd[1:1] = ["-Xptxas", "-v"]
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object in _build/ (in parallel: the
    translation units share no device code) and links the shared library."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ_DIR, exist_ok=True)
    objs = [os.path.join(OBJ_DIR, os.path.basename(s) + ".o") for s in sources()]
    headers = [p for p in deps() if p.endswith((".h", ".cuh"))]
    newest_header = max((os.path.getmtime(p) for p in headers), default=0.0)

    def stale(src: str, obj: str) -> bool:
        if force or not os.path.exists(obj):
            return True
        t = os.path.getmtime(obj)
        return os.path.getmtime(src) > t or newest_header > t

    todo = [(s, o) for s, o in zip(sources(), objs) if stale(s, o)]
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_compile, s, o, verbose) for s, o in todo]:
            f.result()
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp,
                    *objs, "-lpthread"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
