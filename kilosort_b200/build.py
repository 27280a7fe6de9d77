"""Build libks_b200.so in-tree with nvcc for sm_100a.

    python -m kilosort_b200.build

Compiles every ``csrc/*.cu`` into one shared library next to this file
(``kilosort_b200/lib/libks_b200.so``), CUDA runtime linked statically, so the
library loads on a machine without a GPU and exports the C ABI of
``include/ks_b200.h``.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libks_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
         "-fvisibility=hidden", "--expt-relaxed-constexpr", "-cudart", "static"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def build(verbose=False, extra=()):
    os.makedirs(LIB_DIR, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(LIB_DIR, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-I", os.path.join(ROOT, "include"),
               "-dc" if False else "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
