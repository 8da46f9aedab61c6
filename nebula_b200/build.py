"""Build the in-tree CUDA library ``libnbx.so`` and the ``nebula_b200`` CLI.

Everything is compiled for sm_100a with nvcc; the library is written next to
this file so it travels with the source tree (no JIT cache, no site-packages
install)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libnbx.so")
CLI = os.path.join(HERE, "nebula_b200")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_SRCS = ["nbx_api.cpp", "h5lite.cpp", "material.cpp", "octree.cpp"]
CUDA_SRCS = ["transport.cu", "mlp.cu"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.exists(c) or c == "nvcc"):
            return c
    return "nvcc"


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose_ptxas=False, force=False):
    nvcc = _nvcc()
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    inc = ["-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "nbx.h"))
    objs = []
    for src in CUDA_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(obj_dir, src + ".o")
        if force or not _newer(o, [s] + headers):
            flags = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC"] + ARCH
            if verbose_ptxas:
                flags += ["-Xptxas", "-v"]
            _run([nvcc] + flags + inc + ["-c", s, "-o", o])
        objs.append(o)
    for src in HOST_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(obj_dir, src + ".o")
        if force or not _newer(o, [s] + headers):
            _run([nvcc, "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-x", "cu"] + ARCH + inc + ["-c", s, "-o", o])
        objs.append(o)
    if force or not _newer(LIB, objs):
        _run([nvcc, "-shared"] + ARCH + objs + ["-o", LIB])
    main = os.path.join(CSRC, "main.cpp")
    if os.path.exists(main) and (force or not _newer(CLI, [main, LIB] + headers)):
        _run(["g++", "-std=c++17", "-O2"] + inc + [main, "-o", CLI, "-L" + HERE, "-lnbx",
              "-Wl,-rpath,$ORIGIN", "-pthread"])
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv, force="-f" in sys.argv)
