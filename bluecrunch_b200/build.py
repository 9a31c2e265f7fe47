"""Build the in-tree native libraries (no GPU needed; nvcc cross-compiles).

  libbcgpu.so       CUDA engine + C ABI (include/bc_gpu.h), sm_100a only
  libbluecrunch.so  host C: bigfloat API (include/bigfloat.h, include/mul.h)
                    with _fft_mul forwarding to libbcgpu
  bluecrunch        the e-digits command line program

Usage: python -m bluecrunch_b200.build [--force]
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
INC = os.path.join(ROOT, "include")
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")

GPU_LIB = os.path.join(PKG, "libbcgpu.so")
HOST_LIB = os.path.join(PKG, "libbluecrunch.so")
CLI = os.path.join(PKG, "bluecrunch")

NVCC = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
# The image's $CC may point at a gcc without OpenMP; use the system gcc.
GCC = shutil.which("gcc") or "gcc"
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _files(d, exts):
    if not os.path.isdir(d):
        return []
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts))


def build_gpu(force=False):
    srcs = _files(CSRC, (".cu",))
    deps = srcs + _files(CSRC, (".cuh", ".h")) + [os.path.join(INC, "bc_gpu.h")]
    if force or _newer(GPU_LIB, deps):
        _run([NVCC, *GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              "-I" + INC, "-o", GPU_LIB, *srcs, "-lcudart"])
    return GPU_LIB


def build_host(force=False):
    srcs = [f for f in _files(HOST, (".c",)) if not f.endswith("main.c")]
    if not srcs:
        return None
    deps = srcs + _files(HOST, (".h",)) + _files(INC, (".h",)) + [GPU_LIB]
    cflags = ["-std=gnu11", "-O2", "-fPIC", "-fopenmp", "-Wall", "-I" + INC]
    rpath = ["-Wl,-rpath,$ORIGIN"]
    if force or _newer(HOST_LIB, deps):
        _run([GCC, *cflags, "-shared", "-o", HOST_LIB, *srcs, "-L" + PKG, "-lbcgpu", *rpath, "-lm"])
    main = os.path.join(HOST, "main.c")
    if os.path.exists(main) and (force or _newer(CLI, [main, HOST_LIB])):
        _run([GCC, *cflags, "-o", CLI, main, "-L" + PKG, "-lbluecrunch", "-lbcgpu", *rpath, "-lm"])
    return HOST_LIB


def build_all(force=False):
    build_gpu(force)
    build_host(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
