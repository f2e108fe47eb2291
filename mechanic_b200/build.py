"""Build recipe of libmechanic_b200.so (sm_100a, in-tree).

Every translation unit is compiled with IEEE float semantics
(--fmad=false -prec-div=true -prec-sqrt=true -ftz=false) so that the
parity-checked floats are reproducible bit for bit.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_PATH = os.path.join(HERE, "libmechanic_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")
SOURCES = ["mk_api.cu", "mk_step.cu", "mk_sort.cu", "mk_mechanism.cu", "mk_noalloc.cu", "mk_mlp.cu",
           "mk_waits.cu"]
HEADERS = ["mk_device.cuh", "mk_internal.h", "mk_mechanism.h", "mk_mlp.h", "mk_tc.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-DMK_BUILD"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmechanic_b200")
    return path


def sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    deps = sources() + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "mechanic_b200.h"), __file__]
    newest = max(os.path.getmtime(p) for p in deps if os.path.exists(p))
    return os.path.getmtime(LIB_PATH) < newest


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", *objs, "-o", tmp, "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB_PATH)
