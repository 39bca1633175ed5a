"""Builds the sm_100a shared library ``_lib/libddx.so`` from ``csrc/*.cu`` with nvcc.

No GPU is needed to build (nvcc cross-compiles). Objects are rebuilt when a
source or header is newer than the library.
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
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libddx.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-rdc=true", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps() -> list[str]:
    return sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "ddx.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    if up_to_date() and not extra:
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cc = nvcc()
    objs = [os.path.join(OUT_DIR, os.path.basename(src).replace(".cu", ".o")) for src in sources()]

    def compile_one(src: str, obj: str) -> None:
        cmd = [cc, *ARCH, *FLAGS, *(extra or []), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    # the translation units compile independently: one nvcc per host core
    with ThreadPoolExecutor(max_workers=max(1, min(len(objs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(compile_one, src, obj) for src, obj in zip(sources(), objs)]:
            f.result()
    cmd = [cc, *ARCH, "-rdc=true", "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, extra=sys.argv[1:] or None))
