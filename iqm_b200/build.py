"""Builds libiqm_cuda.so (all CUDA sources under csrc/) for sm_100a, in-tree.

    python -m iqm_b200.build            # incremental: rebuilds when a source is newer
    python -m iqm_b200.build --force

The library is compiled with nvcc directly (no torch extension machinery): the product is a
C-ABI shared object declared by include/iqm_cuda.h.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libiqm_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "--threads", "0"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers():
    return glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in sources() + headers())


HOST_SRC = ["methods.cpp", "args.cpp", "png_io.cpp", "image_formats.cpp", "jpeg_decode.cpp", "iqm_cuda.cpp",
            "batch_pipeline.cpp", "main.cpp"]
CUDA_INC = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "include")  # NVTX3 (header-only)
CLI = os.path.join(HERE, "bin", "IQM")
CXX = os.environ.get("IQM_CXX", "/usr/bin/g++")


def build_cli(force=False, verbose=False):
    """Builds the IQM command line (iqm_b200/host) against libiqm_cuda.so."""
    srcs = [os.path.join(HERE, "host", f) for f in HOST_SRC]
    deps = srcs + glob.glob(os.path.join(HERE, "host", "*.h*")) + [LIB]
    if not force and os.path.exists(CLI) and all(os.path.getmtime(f) <= os.path.getmtime(CLI) for f in deps):
        return CLI
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    cmd = [CXX, "-O2", "-std=c++20", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", CUDA_INC, "-o", CLI] + srcs + [
        "-L", HERE, "-liqm_cuda", "-lz", "-ldl", "-pthread", "-Wl,-rpath,$ORIGIN/.."]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return CLI


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    cmd = [NVCC] + ARCH + FLAGS + ["-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "csrc"),
                                   "-shared", "-o", LIB] + sources()
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    build_cli(force="--force" in sys.argv, verbose=True)
