"""Builds charm_b200/libcharm.so: the sm_100a CUDA kernels and the C++ host
runtime behind the C ABI of include/charm_b200.h.

    python charm_b200/build.py

Objects go to charm_b200/_build/; the shared library is written in-tree so
that it ships together with the sources.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcharm.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The CC/CXX of the environment may be wrappers without the system's
# OpenMP and C++ support files, so the system host compiler is used.
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-ccbin", HOST_CXX,
          "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "--expt-relaxed-constexpr"]

SOURCES = ["tables.cu", "shs_grid.cu", "sha_grid.cu", "sctr.cu", "crd.cu", "probe.cu", "rfft.cu", "sha_static.cu", "f32.cu", "shs_tc.cu", "cell.cu", "gfm.cu",
           "engine.cpp", "capi.cpp"]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def compile_one(src, verbose=False):
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC)
                     if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "charm_b200.h"))
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d)
                                   for d in deps):
        return out
    cmd = [nvcc()] + ARCH + COMMON + ["-c", path, "-o", out]
    if src.endswith(".cpp"):
        cmd = [nvcc()] + COMMON + ["-x", "cu", "-c", path, "-o", out] + ARCH
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return out


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, verbose), SOURCES))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(o)
                                   for o in objs):
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-ccbin", HOST_CXX, "-shared", "-o", tmp] + objs + [
        "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
