"""Builds the package's native libraries in-tree (ironav_b200/lib/).

- libironav_inter_cuda.so: the sm_100a kernels and the C ABI of include/ironav_inter.h
  (nvcc -gencode arch=compute_100a,code=sm_100a; nvcc cross-compiles without a GPU).
- libironav_synth.so: the seeded synthetic sequence generator (host C++).
- libironav_inloop_caller.so: a native caller of in-loop mode (host C++ over the CUDA library's C ABI).

Run `python -m ironav_b200.build` (or call build_all()) before importing the bindings.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "lib")
CSRC = os.path.join(PKG, "csrc")

CUDA_LIB = os.path.join(LIB, "libironav_inter_cuda.so")
SYNTH_LIB = os.path.join(LIB, "libironav_synth.so")
INLOOP_LIB = os.path.join(LIB, "libironav_inloop_caller.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3",
]
UNITS = ["ironav_inter.cu", "ironav_batch.cu", "ironav_noalloc.cu", "ironav_stream.cu", "ironav_proposer.cu", "ironav_cabac.cu"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: cannot build the sm_100a kernels")


def _gxx() -> str:
    # the system g++ (an alternative toolchain in $CXX may lack the runtime libraries)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _sources(exts: tuple[str, ...]) -> list[str]:
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(exts)] + [
        os.path.join(ROOT, "include", "ironav_inter.h")
    ]


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    """Compiles each translation unit to an object (in parallel), then links the shared library."""
    deps = _sources((".cu", ".cuh"))
    if force or _stale(CUDA_LIB, deps):
        from concurrent.futures import ThreadPoolExecutor

        os.makedirs(LIB, exist_ok=True)
        objdir = os.path.join(PKG, "_build")
        os.makedirs(objdir, exist_ok=True)

        def compile_unit(u: str) -> str:
            obj = os.path.join(objdir, u.replace(".cu", ".o"))
            cmd = [_nvcc(), *NVCC_FLAGS, *(["-Xptxas=-v"] if verbose else []), "-c", os.path.join(CSRC, u), "-o", obj]
            subprocess.run(cmd, check=True)
            return obj

        with ThreadPoolExecutor(max_workers=len(UNITS)) as pool:
            objs = list(pool.map(compile_unit, UNITS))
        subprocess.run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", CUDA_LIB], check=True)
    return CUDA_LIB


def build_synth(force: bool = False) -> str:
    src = os.path.join(CSRC, "synth.cpp")
    if force or _stale(SYNTH_LIB, [src]):
        os.makedirs(LIB, exist_ok=True)
        subprocess.run([_gxx(), "-O2", "-std=c++17", "-fopenmp", "-shared", "-fPIC", src, "-o", SYNTH_LIB], check=True)
    return SYNTH_LIB


def build_inloop_caller(force: bool = False) -> str:
    """libironav_inloop_caller.so: a native caller of in-loop mode (one thread per slice band), linked
    against the CUDA library (found next to it at run time)."""
    src = os.path.join(CSRC, "inloop_caller.cpp")
    if force or _stale(INLOOP_LIB, [src, CUDA_LIB]):
        subprocess.run([_gxx(), "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread", src, "-L" + LIB, "-lironav_inter_cuda",
                        "-Wl,-rpath,$ORIGIN", "-o", INLOOP_LIB], check=True)
    return INLOOP_LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_synth(force)
    build_cuda(force, verbose)
    build_inloop_caller(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
