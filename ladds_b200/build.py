"""Builds the in-tree native libraries of the package.

* ``ladds_b200/libladds_gpu.so`` -- the sm_100a CUDA kernels and the C ABI of
  ``include/ladds_gpu.h`` (nvcc, ``-gencode arch=compute_100a,code=sm_100a``).
* ``ladds_b200/libladds_population.so`` -- the seeded population generator
  and the population file format alone (g++, no CUDA), for processes that
  must not load GPU code.
* ``ladds_b200/host/libladds_host.so`` -- the C++17 host mirror of the
  reference interface (ladds::Particle, ladds::Integrator,
  ladds::GpuCollisionFunctor, ladds::ConfigReader) on top of the C ABI.

Run ``python -m ladds_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
GPU_LIB = os.path.join(PKG, "libladds_gpu.so")
HOST_DIR = os.path.join(PKG, "host")
HOST_LIB = os.path.join(HOST_DIR, "libladds_host.so")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fopenmp,-O3",
              "-Xptxas", "-O3"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _sources(d, exts):
    out = []
    for dp, _, fs in os.walk(d):
        for f in fs:
            if f.endswith(exts):
                out.append(os.path.join(dp, f))
    return sorted(out)


def build_gpu(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    deps = _sources(CSRC, (".cu", ".cuh", ".cpp", ".h")) + [os.path.join(ROOT, "include", "ladds_gpu.h")]
    if not force and not ptxas_info and _newer(GPU_LIB, deps):
        return GPU_LIB
    cmd = [nvcc(), *NVCC_ARCH, *NVCC_FLAGS, "-shared", "-o", GPU_LIB,
           os.path.join(CSRC, "ladds_gpu.cu"), os.path.join(CSRC, "population.cpp"),
           os.path.join(CSRC, "records_io.cpp"), os.path.join(CSRC, "breakup.cpp"), "-lgomp"]
    if ptxas_info:
        cmd[1:1] = ["-Xptxas", "-v"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if ptxas_info or verbose:
        sys.stdout.write(r.stdout + r.stderr)
    return GPU_LIB


POP_LIB = os.path.join(PKG, "libladds_population.so")


def build_population(force: bool = False, verbose: bool = False) -> str:
    """population.cpp alone as a host library (g++, no CUDA runtime)."""
    srcs = [os.path.join(CSRC, "population.cpp")]
    deps = srcs + [os.path.join(CSRC, "population.h"), os.path.join(CSRC, "physics.cuh"),
                   os.path.join(ROOT, "include", "ladds_gpu.h")]
    if not force and _newer(POP_LIB, deps):
        return POP_LIB
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-o", POP_LIB, *srcs]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("g++ failed:\n" + r.stdout + r.stderr)
    return POP_LIB


PEAKS_LIB = os.path.join(PKG, "libladds_peaks.so")


def build_peaks(force: bool = False, verbose: bool = False) -> str:
    """FMA-pipe throughput diagnostic used by bench.py for the roofline denominators."""
    src = os.path.join(CSRC, "peaks.cu")
    if not force and _newer(PEAKS_LIB, [src]):
        return PEAKS_LIB
    cmd = [nvcc(), *NVCC_ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-o", PEAKS_LIB, src]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    return PEAKS_LIB


def build_host(force: bool = False, verbose: bool = False) -> str:
    srcs = _sources(os.path.join(HOST_DIR, "src"), (".cpp",))
    if not srcs:
        return ""
    deps = srcs + _sources(os.path.join(HOST_DIR, "include"), (".h",)) + [os.path.join(ROOT, "include", "ladds_gpu.h")]
    if not force and _newer(HOST_LIB, deps):
        return HOST_LIB
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", "-I", os.path.join(HOST_DIR, "include"),
           "-I", os.path.join(ROOT, "include"), "-o", HOST_LIB, *srcs, "-L", PKG, "-lladds_gpu",
           "-Wl,-rpath,$ORIGIN/.."]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("g++ failed:\n" + r.stdout + r.stderr)
    return HOST_LIB


HOST_TEST = os.path.join(HOST_DIR, "tests", "test_host")


def build_host_tests(force: bool = False, verbose: bool = False) -> str:
    """The C++ test executable of the host library (tests/test_host_cpp.py runs it)."""
    lib = build_host(force=force, verbose=verbose)
    src = os.path.join(HOST_DIR, "tests", "test_host.cpp")
    if not force and _newer(HOST_TEST, [src, lib]):
        return HOST_TEST
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(HOST_DIR, "include"), "-I",
           os.path.join(ROOT, "include"), "-o", HOST_TEST, src, "-L", HOST_DIR, "-lladds_host", "-L", PKG,
           "-lladds_gpu", f"-Wl,-rpath,{HOST_DIR}", f"-Wl,-rpath,{PKG}"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("g++ failed:\n" + r.stdout + r.stderr)
    return HOST_TEST


def build(force: bool = False, verbose: bool = False) -> None:
    build_gpu(force=force, verbose=verbose)
    build_population(force=force, verbose=verbose)
    build_peaks(force=force, verbose=verbose)
    build_host(force=force, verbose=verbose)
    build_host_tests(force=force, verbose=verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    if "--ptxas" in sys.argv:
        build_gpu(ptxas_info=True)
