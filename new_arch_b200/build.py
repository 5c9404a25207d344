"""Builds libscmf.so and the command-line tools in-tree (new_arch_b200/_lib/).

Kernels are compiled for sm_100a only, with --fmad=false -prec-div=true
-prec-sqrt=true: the move arithmetic must be bit-identical to the CPU oracle,
which is compiled with -ffp-contract=off.  Host C++ is compiled by g++ and the
CUDA runtime is linked statically so the library carries no run-time path
dependency.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(OUT, "obj")
INC = os.path.join(ROOT, "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-std=c++17",
                     "-Xcompiler", "-fPIC", "-I" + INC, "-I" + CSRC] + os.environ.get("SCMF_NVCC_EXTRA", "").split()
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-result", "-ffp-contract=off", "-pthread",
             "-I" + INC, "-I" + CSRC, "-I" + os.path.join(CUDA, "include")]

CU_SOURCES = ["scmf_kernels.cu"]
CXX_SOURCES = ["scmf_engine.cpp", "scmf_api.cpp", "scmf_files.cpp", "scmf_server.cpp", "scmf_state.cpp"]
HEADERS = ["scmf_internal.h", "scmf_math.cuh", "scmf_engine.h"]
TOOLS = {"scmf": "scmf_cli.cpp", "scmf_vtk": "scmf_vtk_cli.cpp"}

LIB = os.path.join(OUT, "libscmf.so")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INC, "scmf.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _newer(o, [s] + hdrs + [__file__]):
            _run([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(OBJ, src + ".o")
        if force or _newer(o, [s] + hdrs + [__file__]):
            _run([CXX] + CXX_FLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-pthread", "-o", LIB] + objs, verbose)
    for tool, src in TOOLS.items():
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        exe = os.path.join(OUT, tool)
        if force or _newer(exe, [s, LIB] + hdrs):
            _run([CXX] + CXX_FLAGS + [s, "-o", exe, "-L" + OUT, "-lscmf", "-Wl,-rpath,$ORIGIN",
                  "-L" + os.path.join(CUDA, "lib64"), "-lcudart_static", "-ldl", "-lrt"], verbose)
    return LIB


def clean() -> None:
    shutil.rmtree(OUT, ignore_errors=True)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
