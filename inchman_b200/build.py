"""Builds the CUDA library of the package (libgpgmp_b200.so) in-tree for sm_100a.

    python -m inchman_b200.build            # incremental
    python -m inchman_b200.build --clean

Every .cu/.cpp under csrc/ becomes one object; the stochastic sampling kernels
are compiled with -fmad=false so their rounding matches a CPU replay.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgpgmp_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(HERE, "..")]
# per-file extra flags
EXTRA = {
    "stochastic.cu": ["-fmad=false"],
    "ensemble.cu": ["-fmad=false"],
    "particles.cu": ["-fmad=false"],
}


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _deps_mtime():
    return max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC)
               if f.endswith((".cuh", ".h")) or f.endswith((".cu", ".cpp")))


def _compile(src: str) -> str:
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    hdr = max([os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
              + [os.path.getmtime(os.path.join(HERE, "..", "include", f))
                 for f in os.listdir(os.path.join(HERE, "..", "include"))])
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), hdr):
        return obj
    cmd = [NVCC, *ARCH, *COMMON, *EXTRA.get(src, []), "-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu", *ARCH, *COMMON, "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(clean: bool = False, verbose: bool = False) -> str:
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(_compile, srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    a = ap.parse_args(argv)
    build(clean=a.clean, verbose=True)


if __name__ == "__main__":
    sys.exit(main())
