"""Build recipe of the native library (nvcc, sm_100a), in-tree.

    python -m localizer_b200.build

produces ``localizer_b200/liblocalizer_b200.so`` next to this file. Objects
are compiled in parallel and rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblocalizer_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
                  "-I" + os.path.join(ROOT, "include")]
SOURCES = ["loc_fit.cu", "loc_capi.cu", "loc_finder.cpp", "loc_synth.cu", "loc_static.cu", "loc_proposal.cu", "loc_finder_gpu.cu", "loc_writer.cpp", "loc_ingest.cu", "loc_mlewg.cu"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".hpp"))]
    hs.append(os.path.join(ROOT, "include", "localizer_b200.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, verbose=False):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + _headers()
    if not _stale(obj, deps):
        return obj
    cmd = [NVCC] + NVFLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    if src == "loc_mlewg.cu":
        # the MLEwG fits follow the reference's FP64 operation order: no contraction into FMA
        cmd.insert(1, "--fmad=false")
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu"] + NVFLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if _stale(LIB, objs):
        # link next to the target and rename: a reader never sees a partly written library
        tmp = LIB + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
