"""Build the sm_100a shared library ``sponge_b200/libsponge_nb.so`` in-tree.

``python -m sponge_b200.build`` (or ``__graft_entry__.build()``) runs nvcc on
every ``csrc/*.cu`` and links them with cuFFT.  nvcc cross-compiles for
sm_100a without a GPU.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsponge_nb.so")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=default", "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale(obj: str, src: str, headers: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + headers)


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(
        os.path.join(CSRC, "*.cuh")) + glob.glob(
        os.path.join(HERE, "..", "include", "*.h"))
    objs = []
    env = dict(os.environ)
    # the toolchain's default host compiler; nvcc picks g++ from PATH
    env.pop("CC", None)
    env.pop("CXX", None)
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if not _stale(obj, src, headers):
            continue
        cmd = [NVCC, *ARCH, *FLAGS, *(extra or []), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd, env=env)
    if not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT)
                                      for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcufft", "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd, env=env)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(OUT)
