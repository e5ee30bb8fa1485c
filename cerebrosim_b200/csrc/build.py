"""Build libcerebrosim_b200.so for sm_100a with nvcc (in-tree, next to the package).

    python -m cerebrosim_b200.csrc.build            # or: from cerebrosim_b200.csrc.build import build; build()

Each .cu is compiled to an object under cerebrosim_b200/_build/ and linked into a shared library with the CUDA
runtime linked statically, so the library needs only the NVIDIA driver at run time and shares the process's
primary context (and therefore device pointers and streams) with PyTorch.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, "libcerebrosim_b200.so")
OBJ = os.path.join(PKG, "_build")
SOURCES = ["capi.cu", "sdf.cu", "lattice_build.cu", "links.cu", "compress.cu", "step.cu", "wss.cu", "gather.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build libcerebrosim_b200.so")
    return exe


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile every CUDA source for sm_100a and link the library; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(HERE, h) for h in os.listdir(HERE) if h.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "cerebrosim.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(HERE, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc()] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", s, "-o", o]
            subprocess.run(cmd, check=True)
    if force or _stale(OUT, objs):
        tmp = OUT + ".tmp"
        subprocess.run([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs, check=True)
        os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
