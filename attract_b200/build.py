"""Build ``libattract_b200.so`` in-tree with nvcc for sm_100a.

    python -m attract_b200.build [--force] [--checked]

``--checked`` builds ``libattract_b200_checked.so`` with -DATT_BOUNDS_CHECK:
every computed grid, list and receptor index of the scoring kernels is
checked before its access; a failed check skips the access and records
(check code, index, bound) for att_kernel_debug_info.  Load it with
$ATTRACT_B200_LIB (the tests do).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = ["score.cu", "build.cu", "allpairs.cu", "capi.cu"]
OUT = os.path.join(HERE, "libattract_b200.so")
OUT_CHECKED = os.path.join(HERE, "libattract_b200_checked.so")
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


def needs_build_checked() -> bool:
    if not os.path.exists(OUT_CHECKED):
        return True
    t = os.path.getmtime(OUT_CHECKED)
    return any(os.path.getmtime(d) > t for d in _inputs()[1])


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    """Compile the CUDA sources into the package directory; returns the .so path."""
    out = OUT_CHECKED if checked else OUT
    if not force and not (needs_build_checked() if checked else needs_build()):
        return out
    nvcc = os.environ.get("NVCC", "nvcc")
    src, _ = _inputs()
    tmp = out + ".tmp"
    cmd = [nvcc, *ARCH, *FLAGS, *(["-DATT_BOUNDS_CHECK"] if checked else []), "-I", os.path.join(ROOT, "include"),
           *src, "-o", tmp]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, checked="--checked" in sys.argv))
