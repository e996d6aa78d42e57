"""Build the hot-path library in tree for sm_100a (nvcc cross-compiles
without a GPU).

    python -m cgd_b200.build        (from cgdycore.jl_b200/)

Two shared libraries come from the same source, both without multiply-add
contraction (-fmad=false):
  libcgd_b200.so        fast build (-DCGD_FAST): the last division of a chain
                        by the time-invariant lumped-mass or Jacobian sum, or
                        by rho, becomes a multiply by a reciprocal computed
                        once per node and level
  libcgd_b200_exact.so  exact build: every division a division; results are
                        bit-identical to the CPU restatement.
Contraction is left off in the fast build too: the balanced initial state
makes the u/v tendencies small residuals of the pressure-gradient and
Coriolis terms, and fused multiply-adds inside the derivative sums of
p ~ 1e5 Pa move them by ~5e-12 relative, beyond the 1e-12 bar.
The host part is compiled with -ffp-contract=off.
"""
import os
import shutil
import subprocess
import sys

from ._lib import LIB_PATH, LIB_PATH_EXACT, PKG_DIR

SRC = os.path.join(PKG_DIR, "csrc", "cgd_b200.cu")
DEPS = [os.path.join(PKG_DIR, "csrc", f) for f in ("cgd_b200.cu", "cgd_kernels.cuh", "cgd_phase2.cuh", "cgd_batch.cuh", "cgd_adjoint.cuh")] + [
    os.path.join(os.path.dirname(PKG_DIR), "include", f) for f in ("cgd_b200.h", "cgd_math.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared"]
VARIANTS = {LIB_PATH: ["-DCGD_FAST", "-fmad=false"], LIB_PATH_EXACT: ["-fmad=false"]}


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise FileNotFoundError("nvcc not found")


def up_to_date(path):
    if not os.path.exists(path):
        return False
    t = os.path.getmtime(path)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force=False, verbose=False):
    procs = []
    for path, extra in VARIANTS.items():
        if not force and up_to_date(path):
            continue
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-o", path, SRC]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd), cmd))
    for p, cmd in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB_PATH)
