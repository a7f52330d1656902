"""Build the in-tree CUDA library ``libpyexner_b200.so`` for sm_100a.

    python -m pyexner_b200.build

Translation units: the float32 kernels, the float64 kernels and the set-up kernels
(both with ``--fmad=false`` so every product and sum rounds on its own, as in the
reference's float64 arithmetic), the C ABI and the allocation-free time step.  Objects
go to ``pyexner_b200/_build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpyexner_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]

UNITS = [
    ("kernels_f32.cu", []),
    ("kernels_f64.cu", ["-fmad=false"]),
    ("setup_f64.cu", ["-fmad=false"]),
    ("kernels_dual.cu", ["-fmad=false"]),
    ("kernels_adj.cu", ["-fmad=false"]),
    ("capi.cu", []),
    ("noalloc.cu", []),
    ("noalloc_f64.cu", ["-fmad=false"]),
]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build pyexner_b200")
    return exe


def sources():
    out = []
    for name in os.listdir(CSRC):
        if name.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, name))
    out.append(os.path.join(os.path.dirname(HERE), "include", "pyexner_b200.h"))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs, cmds = [], []
    knobs = os.environ.get("PXB_NVCC_DEFINES", "").split()  # e.g. "-DPXB_STAGE_MIN_BLOCKS=4" for tuning sweeps
    for src, extra in UNITS:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmds.append([nvcc(), *ARCH, *COMMON, *extra, *knobs, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd))
        for f in [pool.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            f.result()
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
