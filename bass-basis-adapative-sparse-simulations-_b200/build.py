"""Build libbass_b200.so in place (nvcc, sm_100a only).

    python bass-basis-adapative-sparse-simulations-_b200/build.py [--force]

The library is compiled for sm_100a alone (-gencode arch=compute_100a,
code=sm_100a) with -fmad=false so that no double multiply-add is contracted
(the arithmetic must match the CPU oracle bit for bit).  nvcc cross-compiles,
so this runs on a machine without a GPU.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libbass_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-fmad=false", "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-O3"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def deps():
    return sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + \
        glob.glob(os.path.join(HERE, "csrc", "*.h")) + [os.path.join(ROOT, "include", "bass_b200.h")]


def build(force=False, verbose=False):
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps()):
            return LIB
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", LIB] + sources()
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
