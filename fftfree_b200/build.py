"""Builds libfft_cffi.so in-tree (fftfree_b200/lib/) for sm_100a.

CUDA sources go through nvcc with -gencode arch=compute_100a,code=sm_100a;
host C++ through g++; the shared library is linked by nvcc with the static
CUDA runtime.  Only the symbols declared in include/*.h are exported.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libfft_cffi.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["k_common.cu", "k_stft.cu", "k_c2c.cu", "k_cplx.cu", "k_fourstep.cu", "k_grad.cu", "k_ragged.cu", "k_2d.cu", "ft_tools.cu", "meta.cu", "noalloc.cu", "k_tc05.cu"]
CPP_SOURCES = ["abi.cpp", "recovery.cpp", "stream.cpp", "ragged.cpp"]


def _cxx() -> str:
    return shutil.which("g++") or "g++"


def _newer(src_list, target) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hdrs += [os.path.join(REPO, "include", f) for f in os.listdir(os.path.join(REPO, "include"))]
    return hdrs


def _compile(src: str, verbose_ptxas: bool = False) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    path = os.path.join(CSRC, src)
    if not _newer([path] + _deps(), obj):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
               "-c", path, "-o", obj]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = [_cxx(), "-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall",
               f"-I{CUDA_HOME}/include", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"compile failed: {src}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = CU_SOURCES + CPP_SOURCES
    with cf.ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if _newer(objs, LIB):
        cmd = [NVCC, "-shared", *ARCH, "-o", LIB, *objs, "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
