"""Build the in-tree CUDA library hera_b200/libhera_b200.so for sm_100a.

    python -m hera_b200.build [--force]

nvcc compiles csrc/hera_gpu.cu (kernels + the C ABI of include/hera_gpu.h)
into a shared library next to this file; it travels with the source tree
and is what hera_b200.Context loads.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libhera_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("hera_gpu.cu",)]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in ("hera_device.cuh", "hera_batched.cuh", "hera_server.cuh", "hera_fastq.cuh",
                                                                   "hera_classes.cuh", "hera_bam.cuh", "hera_bam_core.h",
                                                                   "hera_bgzf.cuh", "hera_bgzf_core.h")] + [
                  os.path.join(ROOT, "include", "hera_gpu.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-shared", "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    extra = [a for a in sys.argv[1:] if a.startswith("-X")]
    build(force="--force" in sys.argv, verbose=True, extra=extra)
