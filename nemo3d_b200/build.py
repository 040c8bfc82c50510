"""Compile libtbgpu.so (CUDA sm_100a) in-tree with nvcc."""

from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtbgpu.so")
SOURCES = ["topology.cu", "build.cu", "spmv.cu", "spmv_async.cu", "lanczos.cu", "capi.cu",
           "noalloc.cu", "band_eig.cu", "blk_lanczos.cu", "spmm_async.cu", "io.cu",
           "recompute.cu", "optics.cu", "vff.cu",
           "batch.cu", "spmv_tile.cu", "warmstart.cu", "spmv_lane.cu", "spmv_pen.cu", "bdots_tc.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
              "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = glob.glob(os.path.join(CSRC, "*")) + [
        os.path.join(HERE, "..", "include", "tbgpu.h")]
    return all(os.path.getmtime(p) <= t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [_nvcc()] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
