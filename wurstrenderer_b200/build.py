"""Build recipe for the native library and CLI (sm_100a only).

Produces, in this package directory:
  libwurst_b200.so   C ABI of include/wurst_b200.h (host C++ + CUDA kernels)
  wurst_b200         command-line front end (--simple2parse / --jsimple2parse)

Objects go to ``_build/``; a source is recompiled only when it (or a header)
is newer than its object. Run ``python -m wurstrenderer_b200.build``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libwurst_b200.so")
CLI = os.path.join(PKG, "wurst_b200")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3,-Wall,-Wno-unused-function",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]
CU_FLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-O3"]

SOURCES = ["wr_scene_io.cpp", "wr_image_io.cpp", "wr_bvh.cpp", "wr_capi.cpp", "wr_kernels.cu", "wr_noalloc.cu", "wr_lbvh.cu", "wr_guide.cu"]


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max(os.path.getmtime(h) for h in hs)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = _newest_header()
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(path), hdr):
            # .cpp sources go through nvcc too so that every object shares one toolchain
            if src.endswith(".cu") or src == "wr_capi.cpp":
                flags = CU_FLAGS + ["-x", "cu"]
            else:
                flags = ARCH + COMMON + ["-x", "c++"]
            _run([NVCC] + flags + ["-c", path, "-o", obj], verbose)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fPIC", "-lpthread", "-lz"], verbose)
    cli_src = os.path.join(CSRC, "wr_cli.cpp")
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(LIB), os.path.getmtime(cli_src)):
        _run([NVCC] + ARCH + ["-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-x", "c++", cli_src, "-o", CLI,
              "-L", PKG, "-lwurst_b200", "-Xlinker", "-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
