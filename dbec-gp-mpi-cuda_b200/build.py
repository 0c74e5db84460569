"""Build recipe of the B200 solver library and its command-line programs.

Compiles, for sm_100a only:
  lib/libgpe.so            C ABI (include/gpe.h): kernels + handle
  lib/libgpe_cufft.so      cuFFT convolution kept as a timed comparison (include/gpe_cufft.h)
  bin/imag3d-mpicuda       drop-in CLI for imaginary time
  bin/real3d-mpicuda       drop-in CLI for real time
Uses nvcc directly (no torch extension): the library has no torch types in
its interface.  Outputs stay inside the package directory so they travel with
the repository snapshot.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
LIB_DIR = os.path.join(PKG, "lib")
BIN_DIR = os.path.join(PKG, "bin")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                  "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]

LIB_SOURCES = ["solver.cu", "noalloc.cu", "batch.cu", "server.cpp"]
LIB_DEPS = LIB_SOURCES + ["common.cuh", "fft.cuh", "kernels.cuh", "step_kernels.cuh", "sweep_kernels.cuh", "tma.cuh",
                          "batch_kernels.cuh", "internal.h"]
OBJ_DIR = os.path.join(PKG, "_build")
HOST_COMMON = ["cfg.cpp", "cli.cpp"]
PROGRAMS = {"imag3d-mpicuda": "imag3d_main.cpp", "real3d-mpicuda": "real3d_main.cpp"}

LIB = os.path.join(LIB_DIR, "libgpe.so")
# the cuFFT pipeline kept only as a timed comparison: its own library, so the
# solver itself never links cuFFT
CUFFT_SOURCES = ["cufft_compare.cu"]
CUFFT_LIB = os.path.join(LIB_DIR, "libgpe_cufft.so")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_lib(force=False, verbose_ptxas=False):
    """Compiles the library's translation units in parallel (each depends on
    its source and every header, so a header change rebuilds them all), then
    links."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in LIB_DEPS] + [os.path.join(INCLUDE, "gpe.h")]
    if not (force or _stale(LIB, deps)):
        return LIB
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    objs = [os.path.join(OBJ_DIR, f + ".o") for f in LIB_SOURCES]
    headers = [d for d in deps if not d.endswith((".cu", ".cpp"))]
    jobs = [[NVCC] + NVFLAGS + extra + ["-c", "-o", o, os.path.join(CSRC, f)]
            for f, o in zip(LIB_SOURCES, objs) if force or _stale(o, headers + [os.path.join(CSRC, f)])]
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(_run, jobs))
    _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"])
    return LIB


def build_cufft_lib(force=False):
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in CUFFT_SOURCES] + [os.path.join(INCLUDE, "gpe.h"),
                                                             os.path.join(INCLUDE, "gpe_cufft.h")]
    if force or _stale(CUFFT_LIB, deps):
        _run([NVCC] + NVFLAGS + ["-shared", "-o", CUFFT_LIB] + [os.path.join(CSRC, f) for f in CUFFT_SOURCES] +
             ["-lcufft", "-lcudart"])
    return CUFFT_LIB


def build_programs(force=False):
    os.makedirs(BIN_DIR, exist_ok=True)
    out = {}
    common = [os.path.join(HOST, f) for f in HOST_COMMON]
    for name, main in PROGRAMS.items():
        target = os.path.join(BIN_DIR, name)
        srcs = common + [os.path.join(HOST, main)]
        deps = srcs + [os.path.join(HOST, "cfg.h"), os.path.join(HOST, "cli.h"), LIB]
        if force or _stale(target, deps):
            _run(["g++", "-O2", "-std=c++17", "-I" + INCLUDE, "-I" + HOST, "-o", target] + srcs +
                 ["-L" + LIB_DIR, "-lgpe", "-Wl,-rpath,$ORIGIN/../lib"])
        out[name] = target
    return out


def build(force=False):
    build_lib(force)
    build_cufft_lib(force)
    if os.path.exists(os.path.join(HOST, "cli.cpp")):
        build_programs(force)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
