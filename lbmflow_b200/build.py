"""Compile the sm_100a CUDA library in-tree (lbmflow_b200/_build/liblbmb.so).

Each translation unit (one engine instantiation per lattice and storage
type, the C ABI, the allocation-free entry point, the host geometry) is
compiled by its own nvcc process in parallel and then linked.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "liblbmb.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def units():
    return sorted(os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".h"))]
    return hs + [os.path.join(HERE, "..", "include", "lbmb.h"), __file__]


def _obj(u):
    return os.path.join(OBJ_DIR, os.path.basename(u) + ".o")


def _stale(u, newest_header):
    o = _obj(u)
    return not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(u), newest_header)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    newest_header = max(os.path.getmtime(h) for h in headers())
    todo = [u for u in units() if force or _stale(u, newest_header)]
    flags = NVCC_FLAGS + list(extra_flags or [])

    def compile_one(u):
        cmd = [nvcc] + flags + ["-c", u, "-o", _obj(u) + ".tmp"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {u}:\n{r.stderr}")
        os.replace(_obj(u) + ".tmp", _obj(u))
        return u

    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            list(ex.map(compile_one, todo))
    objs = [_obj(u) for u in units()]
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
