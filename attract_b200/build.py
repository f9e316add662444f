"""Build ``libattract_b200.so`` in-tree with nvcc for sm_100a.

    python -m attract_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = ["score.cu", "build.cu", "allpairs.cu", "capi.cu"]
OUT = os.path.join(HERE, "libattract_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def _inputs():
    src = [os.path.join(HERE, "csrc", s) for s in SOURCES]
    deps = src + [os.path.join(HERE, "csrc", "common.cuh"), os.path.join(ROOT, "include", "attract_b200.h")]
    return src, deps


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(d) > t for d in _inputs()[1])


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the CUDA sources into the package directory; returns the .so path."""
    if not force and not needs_build():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    src, _ = _inputs()
    tmp = OUT + ".tmp"
    cmd = [nvcc, *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), *src, "-o", tmp]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
