"""The allocation-free Jacobian + Schur solve (cgd_jac_schur_solve_noalloc),
for callers whose device memory belongs to their own pool allocator and who
cannot let the library call cudaMalloc.  It is called through the C ABI on
device buffers and checked against the handle-based cgd_jac +
cgd_schur_solve on the same inputs, two calls in a row (the second reuses
the static band scratch the first one filled).  The call only enqueues on
the given stream, so the test synchronises before it reads the results.
Collected last so it also runs after every other GPU test in the same
process."""
import ctypes

import numpy as np
import pytest

from _cases import make_case, rel_err_per_field

pytestmark = pytest.mark.gpu


def _cfg(g, NumTr, phys):
    from cgd_b200 import _lib
    c = _lib.CgdConfig()
    c.OrdPoly, c.nz, c.NumTr, c.NF, c.NumG = g.OrdPoly, g.nz, NumTr, g.NF, g.NumG
    c.Grav, c.Rd, c.Cpd, c.p0, c.Omega = phys.Grav, phys.Rd, phys.Cpd, phys.p0, phys.Omega
    return c


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).transpose(*reversed(range(a.ndim))))).cuda()


def _host(t):
    return t.cpu().numpy().transpose(*reversed(range(t.dim())))


@pytest.mark.parametrize("exact", [False, True])
def test_noalloc_matches_handle_solve_twice(oracle_mod, built_lib, cuda_ok, exact):
    import torch
    from cgd_b200 import Dycore, _lib
    from cgd_b200.physics import PhysParameters
    L = _lib.lib(exact=exact)
    phys = PhysParameters()
    o, g, U, nu = make_case(oracle_mod, 4, 4, 20, 1, "quadratic")
    d = Dycore(g, 1, nu, exact=exact)
    cfg = _cfg(g, 1, phys)
    rng = np.random.default_rng(5)
    dz_t = _dev(g.dz)
    k_t = torch.empty(U.shape[::-1], dtype=torch.float64, device="cuda")
    for call, fac in enumerate((300.0, 120.0)):
        Ui = U * (1.0 + 1e-3 * call)
        Ui = np.asfortranarray(Ui)
        v = np.asfortranarray(rng.standard_normal(U.shape))
        d.jac(Ui)
        v_ref = v.copy(order="F")
        k_ref = d.schur_solve(v_ref, fac)
        U_t, v_t = _dev(Ui), _dev(v)
        k_t.fill_(np.nan)
        torch.cuda.synchronize()
        rc = L.cgd_jac_schur_solve_noalloc(ctypes.byref(cfg), U_t.data_ptr(), dz_t.data_ptr(), k_t.data_ptr(),
                                           v_t.data_ptr(), fac, None)
        assert rc == 0, (rc, L.cgd_strerror(rc))
        torch.cuda.synchronize()
        k_g, v_g = _host(k_t), _host(v_t)
        assert rel_err_per_field(k_g, k_ref).max() <= 1e-12
        assert rel_err_per_field(v_g, v_ref).max() <= 1e-12
        assert np.array_equal(k_g, k_ref) and np.array_equal(v_g, v_ref)   # same kernels, same order
    d.close()


def test_noalloc_rejects_oversize(built_lib, cuda_ok):
    import torch
    from cgd_b200 import _lib
    from cgd_b200.physics import PhysParameters
    L = _lib.lib()
    phys = PhysParameters()
    c = _lib.CgdConfig()
    c.OrdPoly, c.nz, c.NumTr, c.NF = 4, 64, 0, 6
    c.NumG = _lib.NOALLOC_SCRATCH_DOUBLES // (8 * 63) + 1
    c.Grav, c.Rd, c.Cpd, c.p0 = phys.Grav, phys.Rd, phys.Cpd, phys.p0
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = t.data_ptr()
    assert L.cgd_jac_schur_solve_noalloc(ctypes.byref(c), p, p, p, p, 100.0, None) == -2
