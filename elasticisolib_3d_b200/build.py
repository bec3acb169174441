"""Build the native library libelastic3d_b200.so in-tree for sm_100a.

The library holds the CUDA kernels, the engine, the C ABI declared in
include/elastic3d_b200.h and the native host preparation routines.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libelastic3d_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["engine.cu", "c_abi.cpp", "host_prep.cpp"]
HEADERS = ["common.cuh", "kernels.cuh", "engine.h", "schedule.h", "shot_operators.cpp"]


def _host_compiler():
    # /usr/bin/g++ ships the OpenMP runtime spec; some environments put a
    # g++ without it first on PATH.
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")


def _operators_module():
    import sysconfig
    return os.path.join(HERE, "pyElastic_iso_float_3D" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def _stale():
    if not os.path.exists(LIB) or not os.path.exists(_operators_module()):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "elastic3d_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    ccbin = _host_compiler()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".", "_") + ".o")
        cmd = [nvcc, "-c", os.path.join(CSRC, src), "-o", obj, "-O3", "-std=c++17", "-lineinfo",
               "-Xcompiler", "-fPIC,-fopenmp", "-ccbin", ccbin] + ARCH
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        else:
            cmd = [nvcc, "-x", "c++", "-c", os.path.join(CSRC, src), "-o", obj, "-O3", "-std=c++17",
                   "-Xcompiler", "-fPIC,-fopenmp", "-ccbin", ccbin] + ARCH
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", "-o", tmp] + objs + ARCH + ["-ccbin", ccbin, "-Xcompiler", "-fopenmp", "-lgomp",
                                                         "-lcudart"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    build_operators(ccbin, verbose)
    return LIB


def build_operators(cxx=None, verbose=False):
    """The pybind11 module of the C++ shot operators (csrc/shot_operators.cpp), linked against the
    library above and loaded from the package directory."""
    import sysconfig

    import pybind11
    cxx = cxx or _host_compiler()
    out = _operators_module()
    cmd = [cxx, "-O3", "-shared", "-fPIC", "-fvisibility=hidden", "-std=c++17", "-I" + pybind11.get_include(),
           "-I" + sysconfig.get_paths()["include"], "-I" + os.path.join(HERE, "..", "include"),
           os.path.join(CSRC, "shot_operators.cpp"), "-L" + HERE, "-lelastic3d_b200", "-Wl,-rpath,$ORIGIN",
           "-o", out + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
