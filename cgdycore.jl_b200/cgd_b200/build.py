"""Build libcgd_b200.so in tree for sm_100a (nvcc cross-compiles without a GPU).

    python -m cgd_b200.build        (from cgdycore.jl_b200/)

-fmad=false keeps every device multiply and add separately rounded, which is
what makes the kernels bit-identical to the CPU restatement; the host part
is compiled with -ffp-contract=off for the same reason.
"""
import os
import shutil
import subprocess
import sys

from ._lib import LIB_PATH, PKG_DIR

SRC = os.path.join(PKG_DIR, "csrc", "cgd_b200.cu")
DEPS = [os.path.join(PKG_DIR, "csrc", f) for f in ("cgd_b200.cu", "cgd_kernels.cuh", "cgd_mixed.cuh")] + [
    os.path.join(os.path.dirname(PKG_DIR), "include", f) for f in ("cgd_b200.h", "cgd_math.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared"]


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise FileNotFoundError("nvcc not found")


def up_to_date():
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB_PATH
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB_PATH, SRC]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB_PATH)
