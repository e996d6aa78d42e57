"""CPU tests of the C ABI surface and of the shared elementary functions.

* libcgd_b200.so builds for sm_100a here (nvcc cross-compiles), loads, and
  exports every function declared in include/cgd_b200.h; argument checks
  return the documented codes without touching a GPU.
* cgd_exp / cgd_log (include/cgd_math.h) stay within 2 ulp of the C library.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cgd_[a-z0-9_]+)\s*\(", txt)))


@pytest.mark.parametrize("exact", [False, True])
def test_library_exports_every_declared_symbol(built_lib, exact):
    from cgd_b200 import _lib
    path = _lib.LIB_PATH_EXACT if exact else _lib.LIB_PATH
    L = ctypes.CDLL(path)
    names = _declared("cgd_b200.h")
    assert names, "no declarations parsed"
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/cgd_b200.h but not exported"
    assert set(names) == set(_lib.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


def test_library_is_sm100a(built_lib):
    """The build command targets compute_100a/sm_100a (no PTX for other archs)."""
    from cgd_b200 import build
    flags = " ".join(build.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags
    # the forward kernels without multiply-add contraction (the exact build
    # matches the restatement bit for bit), the adjoint's unit with it
    assert build.VARIANTS[build.LIB_PATH_EXACT] == [] and build.FWD_FLAGS == ["-fmad=false"]
    assert build.ADJ_FLAGS == ["-fmad=true"]
    from cgd_b200 import _lib
    assert b"sm_100a" in _lib.lib().cgd_version() and b"fast" in _lib.lib().cgd_version()
    assert b"exact" in _lib.lib(exact=True).cgd_version()


def test_argument_errors_without_device(built_lib):
    from cgd_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    # null config
    assert L.cgd_create(None, *([None] * 8), ctypes.byref(h)) == -1
    cfg = _lib.CgdConfig()
    cfg.OrdPoly, cfg.nz, cfg.NumTr, cfg.NF, cfg.NumG = 9, 10, 0, 6, 26
    cfg.Grav, cfg.Rd, cfg.Cpd, cfg.p0 = 9.8, 287.0, 1004.0, 1e5
    assert L.cgd_create(ctypes.byref(cfg), *([None] * 8), ctypes.byref(h)) == -7   # p > 4
    cfg.OrdPoly = 4
    cfg.nz = 100
    assert L.cgd_create(ctypes.byref(cfg), *([None] * 8), ctypes.byref(h)) == -7   # nz > 64
    cfg.nz = 10
    assert L.cgd_create(ctypes.byref(cfg), *([None] * 8), ctypes.byref(h)) == -1   # null arrays
    for f in ("cgd_rhs", "cgd_prepare", "cgd_jac"):
        assert getattr(L, f)(None, None, None) == -1
    assert L.cgd_ros_step(None, None, 1.0, 1) == -1
    assert L.cgd_strerror(-4) == b"non-finite value in the state"


def test_create_without_device_reports_no_device(built_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from cgd_b200 import _lib
    L = _lib.lib()
    cfg = _lib.CgdConfig()
    cfg.OrdPoly, cfg.nz, cfg.NumTr, cfg.NF, cfg.NumG = 1, 2, 0, 6, 8
    cfg.Grav, cfg.Rd, cfg.Cpd, cfg.p0 = 9.8, 287.0, 1004.0, 1e5
    glob = np.zeros(24, np.int64) + 1
    arr = np.zeros(10000)
    h = ctypes.c_void_p()
    rc = L.cgd_create(ctypes.byref(cfg), glob.ctypes.data, *([arr.ctypes.data] * 7), ctypes.byref(h))
    assert rc in (-8, -6)


def test_elementary_functions_within_two_ulp(tmp_path):
    src = tmp_path / "m.c"
    src.write_text('#include "cgd_math.h"\n'
                   "void f(int which, const double *x, double *y, int n){\n"
                   " for(int i=0;i<n;i++) y[i] = which==0 ? cgd_exp(x[i]) : which==1 ? cgd_log(x[i]) :"
                   " cgd_pow(x[i], 0.4);}\n")
    so = tmp_path / "m.so"
    subprocess.run(["/usr/bin/gcc", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I",
                    os.path.join(ROOT, "include"), "-o", str(so), str(src), "-lm"], check=True)
    L = ctypes.CDLL(str(so))
    L.f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]

    def run(which, x):
        y = np.zeros_like(x)
        L.f(which, x.ctypes.data, y.ctypes.data, x.size)
        return y

    def ulps(a, b):
        return np.abs(a.view(np.int64) - b.view(np.int64))

    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-700, 700, 200000), rng.uniform(-1, 1, 200000)])
    assert ulps(run(0, x), np.exp(x)).max() <= 2
    x = np.concatenate([rng.uniform(1e-6, 10, 200000), rng.uniform(0.5, 1.5, 200000),
                        np.exp(rng.uniform(-600, 600, 20000))])
    assert ulps(run(1, x), np.log(x)).max() <= 2
    x = rng.uniform(0.01, 2.0, 100000)
    ref = np.power(x, 0.4)
    assert (np.abs(run(2, x) - ref) / ref).max() < 1e-15
    assert run(0, np.array([1000.0]))[0] == np.inf and run(1, np.array([0.0]))[0] == -np.inf
