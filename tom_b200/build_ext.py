"""Build libtomgpu.so (sm_100a) in-tree from tom_b200/csrc with nvcc.

Objects go to tom_b200/_build/, the library to tom_b200/libtomgpu.so.  Each
translation unit compiles in its own nvcc process; the link uses the static
CUDA runtime so the library does not depend on which libcudart a host process
(e.g. torch) has loaded.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtomgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I" + SRC, "-I" + os.path.join(os.path.dirname(HERE), "include")]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(SRC) if f.endswith((".cu", ".cpp")))


def _newer(src_paths, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in src_paths)


def _headers():
    return [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".h", ".cuh"))] + [
        os.path.join(os.path.dirname(HERE), "include", "tomgpu.h")]


def compile_one(src: str, verbose: bool) -> str:
    os.makedirs(BUILD, exist_ok=True)
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(SRC, src)
    if not _newer([path] + _headers(), obj):
        return obj
    cmd = [nvcc()] + ARCH + COMMON + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd[1:1] = ["-x", "cu"] if False else []
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> str:
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: compile_one(s, verbose), srcs))
    if _newer(objs, LIB):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
