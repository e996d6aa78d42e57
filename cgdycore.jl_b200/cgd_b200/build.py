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
The adjoint kernels (csrc/cgd_adjoint.cu) are a second translation unit,
compiled with contraction in both libraries: they are checked against finite
differences, not bit for bit.  The two objects are linked into one library.
The host part is compiled with -ffp-contract=off.
"""
import os
import shutil
import subprocess
import sys

from ._lib import LIB_PATH, LIB_PATH_EXACT, PKG_DIR

SRC = os.path.join(PKG_DIR, "csrc", "cgd_b200.cu")
SRC_ADJ = os.path.join(PKG_DIR, "csrc", "cgd_adjoint.cu")
OBJ_DIR = os.path.join(PKG_DIR, "_build")
DEPS = [os.path.join(PKG_DIR, "csrc", f) for f in ("cgd_b200.cu", "cgd_adjoint.cu", "cgd_kernels.cuh", "cgd_phase2.cuh",
                                                   "cgd_batch.cuh", "cgd_adjoint.cuh", "cgd_adjoint_launch.h")] + [
    os.path.join(os.path.dirname(PKG_DIR), "include", f) for f in ("cgd_b200.h", "cgd_math.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-ffp-contract=off"]
# (nvcc --split-compile builds about three times faster here but its code is
# slower: the tendency kernel took 1.52 instead of 1.41 ms per launch)
VARIANTS = {LIB_PATH: ["-DCGD_FAST"], LIB_PATH_EXACT: []}
FWD_FLAGS = ["-fmad=false"]   # the forward translation unit (cgd_b200.cu)
ADJ_FLAGS = ["-fmad=true"]    # the adjoint translation unit (cgd_adjoint.cu)


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


def _run_all(cmds, verbose):
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd), cmd))
    for p, cmd in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)


def build(force=False, verbose=False):
    os.makedirs(OBJ_DIR, exist_ok=True)
    todo = [(path, extra) for path, extra in VARIANTS.items() if force or not up_to_date(path)]
    comp, link = [], []
    for path, extra in todo:
        tag = os.path.splitext(os.path.basename(path))[0]
        o_fwd = os.path.join(OBJ_DIR, tag + "_fwd.o")
        o_adj = os.path.join(OBJ_DIR, tag + "_adj.o")
        xv = ["-Xptxas=-v"] if verbose else []
        comp.append([nvcc()] + NVCC_FLAGS + extra + xv + FWD_FLAGS + ["-c", "-o", o_fwd, SRC])
        comp.append([nvcc()] + NVCC_FLAGS + extra + xv + ADJ_FLAGS + ["-c", "-o", o_adj, SRC_ADJ])
        link.append([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", path, o_fwd, o_adj])
    _run_all(comp, verbose)
    _run_all(link, verbose)
    shutil.rmtree(OBJ_DIR, ignore_errors=True)   # the objects live on inside the libraries
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB_PATH)
