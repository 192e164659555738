"""Build libsmmp_b200.so (sm_100a kernels + host runtime + C ABI) in-tree.

    python smmp-svn_b200/build.py          # incremental
    python smmp-svn_b200/build.py --force  # rebuild everything

Objects go to smmp-svn_b200/_build/, the library to
smmp-svn_b200/smmp/libsmmp_b200.so next to the Python package that loads it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "smmp", "libsmmp_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                  "-I" + SRC, "-I" + INCLUDE]
# host set-up code keeps separately rounded FP64 arithmetic (no contraction)
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I" + SRC, "-I" + INCLUDE]

CUDA_SOURCES = ["kernels.cu", "runtime.cu", "capi.cu", "surrogate.cu", "esolan.cu"]
# the analytic SASA keeps the reference's separately rounded FP64 arithmetic
CUDA_EXTRA = {"esolan.cu": ["-fmad=false"]}
CXX_SOURCES = ["molbuild.cpp", "ecepp.cpp", "topology.cpp", "muca.cpp", "minimize.cpp"]


def _headers():
    return [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".hpp", ".cuh", ".h"))] + \
        [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(force=False, verbose_ptxas=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    objs = []
    for f in CUDA_SOURCES:
        src = os.path.join(SRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            _run([NVCC] + NVFLAGS + CUDA_EXTRA.get(f, []) + extra + ["-c", src, "-o", obj])
    # the sweep kernels again with 384 threads per chain (small molecules)
    src = os.path.join(SRC, "kernels.cu")
    obj = os.path.join(OBJ, "kernels_t384.cu.o")
    objs.append(obj)
    if force or _stale(obj, [src] + hdrs):
        extra = ["-Xptxas", "-v"] if verbose_ptxas else []
        _run([NVCC] + NVFLAGS + ["-DSMMP_THREADS=384", "-DSMMP_BLOCK_VARIANT=t384"] + extra +
             ["-c", src, "-o", obj])
    for f in CXX_SOURCES:
        src = os.path.join(SRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            _run([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
