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
    "individual.cu": ["-fmad=false"],
}


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


# device headers that csrc/jit.cpp compiles again at run time (NVRTC), embedded as
# string literals in the generated csrc/_jit_sources.h
JIT_HEADERS = [("common.cuh", os.path.join(CSRC, "common.cuh")),
               ("stoch_device.cuh", os.path.join(CSRC, "stoch_device.cuh")),
               ("individual_device.cuh", os.path.join(CSRC, "individual_device.cuh")),
               ("../../include/gpgmp_c.h", os.path.join(HERE, "..", "include", "gpgmp_c.h"))]
JIT_OUT = os.path.join(CSRC, "_jit_sources.h")


def _gen_jit_sources():
    parts = ["// Generated by inchman_b200/build.py from the device headers; do not edit.",
             "#pragma once", "namespace gpgmp {",
             f"constexpr int kJitHeaderCount = {len(JIT_HEADERS)};",
             "static const char* const kJitHeaderNames[] = {" +
             ", ".join(f'"{n}"' for n, _ in JIT_HEADERS) + "};",
             "static const char* const kJitHeaderSources[] = {"]
    for name, path in JIT_HEADERS:
        text = open(path).read()
        if ")GPGMPJIT\"" in text:
            raise RuntimeError(f"{path} contains the raw-string delimiter")
        parts.append(f'R"GPGMPJIT({text})GPGMPJIT",')
    parts += ["};", "}  // namespace gpgmp", ""]
    out = "\n".join(parts)
    if not os.path.exists(JIT_OUT) or open(JIT_OUT).read() != out:
        with open(JIT_OUT, "w") as f:
            f.write(out)


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
    _gen_jit_sources()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(_compile, srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    # NVRTC and the driver API are opened with dlopen on first use (csrc/jit.cpp)
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
