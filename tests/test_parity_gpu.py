"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the
same seeded inputs.

Bars (from the hot-path contract):
  * index/DSS maps bit-exact (checked on the CPU side in test_golden_grid);
  * FP64 tendencies within 1e-12 relative max-norm per field;
  * the state after 10 Rosenbrock-W steps within 1e-10.
Two builds are checked.  The exact build evaluates the reference's
expressions in the same order without contraction and sums the DSS in the
oracle's order, so its results are asserted bit-identical.  The fast build
(reciprocal multiplies by time-invariant sums, the warp-scan tridiagonal
solve; no contraction either) is held to the tolerances.
"""
import numpy as np
import pytest

from _cases import make_case, rel_err_per_field

pytestmark = pytest.mark.gpu

TOL_RHS = 1e-12
TOL_STEP = 1e-10


@pytest.fixture(scope="module")
def lib_ready(built_lib, cuda_ok):
    return True


def _dycore(grid, NumTr, nu, **kw):
    from cgd_b200 import Dycore
    return Dycore(grid, NumTr, nu, **kw)


def _same(a, b, exact, tol):
    """Bit-identical for the exact build, within tol (relative max-norm per
    field) for the fast build."""
    err = rel_err_per_field(a, b)
    assert err.max() <= tol, err
    if exact:
        assert np.array_equal(a, b), err


CASES = {
    "small": dict(nPanel=6, p=4, nz=10, NumTr=0, stretch="uniform"),
    "tracers_p3": dict(nPanel=5, p=3, nz=12, NumTr=2, stretch="quadratic"),
    "nz64": dict(nPanel=4, p=4, nz=64, NumTr=1, stretch="quadratic"),
    "p2": dict(nPanel=6, p=2, nz=7, NumTr=0, stretch="uniform"),
    # edge cases: p = 1 (eight levels per warp), three layers (the upwind
    # stencil clamped at both ends of every interface), the maximum of four
    # tracers, the maximum of 64 levels at p = 2
    "p1": dict(nPanel=5, p=1, nz=9, NumTr=1, stretch="quadratic"),
    "nz3": dict(nPanel=4, p=4, nz=3, NumTr=0, stretch="uniform"),
    "tracers4": dict(nPanel=3, p=4, nz=17, NumTr=4, stretch="quadratic"),
    "p2_nz64": dict(nPanel=3, p=2, nz=64, NumTr=0, stretch="quadratic"),
}


@pytest.fixture(scope="module", params=[(c, v) for c in CASES for v in ("exact", "fast")],
                ids=lambda p: f"{p[0]}-{p[1]}")
def case(request, oracle_mod, lib_ready):
    name, variant = request.param
    c = CASES[name]
    o, g, U, nu = make_case(oracle_mod, c["nPanel"], c["p"], c["nz"], c["NumTr"], c["stretch"])
    d = _dycore(g, c["NumTr"], nu, exact=(variant == "exact"))
    yield name, o, g, U, nu, d
    d.close()


def test_pressure(case):
    name, o, g, U, nu, d = case
    pg, po = d.fcn_prepare(U), o.pressure(U)
    assert np.abs(pg - po).max() <= 1e-15 * np.abs(po).max()
    if d.exact:
        assert np.array_equal(pg, po)


def test_hypervisc_phase1(case):
    """The phase-1 cache holds second derivatives of theta = rho*theta/rho
    (~300 K with 1e-2 K structure), so any change of rounding moves it by
    ~1e-12 of its own scale; the fast build is held to 1e-11 here and to the
    1e-12 bar on the tendency it feeds (test_rhs)."""
    name, o, g, U, nu, d = case
    _same(d.hypervisc_phase1(U), o.hypervisc1(U), d.exact, TOL_RHS if d.exact else 1e-11)


def test_rhs(case):
    name, o, g, U, nu, d = case
    _same(d.fcn(U), o.rhs(U), d.exact, TOL_RHS)


def test_jacobian_and_schur(case):
    name, o, g, U, nu, d = case
    bo = o.jac(U)
    bg = d.jac(U)
    assert np.abs(bg - bo).max() <= 1e-14 * np.abs(bo).max()
    rng = np.random.default_rng(11)
    v = np.asfortranarray(rng.standard_normal(U.shape))
    ko, vo = o.schur(v, 300.0)
    vg = v.copy(order="F")
    kg = d.schur_solve(vg, 300.0)
    _same(kg, ko, d.exact, TOL_RHS)
    _same(vg, vo, d.exact, TOL_RHS)
    if d.exact:
        assert np.array_equal(bg, bo)


def test_jcache_bands_and_explicit_solve(case):
    """Per-function injection as the reference's RosenbrockSchur! does it:
    JacSchurGPU!(J, U, ...) fills the caller's four JCache band arrays
    (cgd_jac_bands), then SchurSolveGPU!(k, v, J, fac, ...) reads them
    (cgd_schur_solve_bands), on host arrays and on device tensors.  The
    bands match the oracle's Jacobian and the solve its Schur solve."""
    import torch
    name, o, g, U, nu, d = case
    bo = o.jac(U)                       # (4, 2, nz-1, NumG)
    J = d.jac_bands(d.new_bands(), U)
    for i in range(4):
        assert np.abs(J[i] - bo[i]).max() <= 1e-14 * np.abs(bo).max()
        if d.exact:
            assert np.array_equal(J[i], bo[i])
    rng = np.random.default_rng(12)
    v = np.asfortranarray(rng.standard_normal(U.shape))
    ko, vo = o.schur(v, 120.0)
    d.jac(U * 1.01)                     # the handle's own bands now differ
    vg = v.copy(order="F")
    kg = d.schur_solve_bands(d.new_state(), vg, J, 120.0)
    _same(kg, ko, d.exact, TOL_RHS)
    _same(vg, vo, d.exact, TOL_RHS)
    # device arrays: bands and state as CUDA tensors, read in place
    Jt = [torch.from_numpy(np.ascontiguousarray(b.transpose(2, 1, 0))).cuda() for b in J]
    vt = torch.from_numpy(np.ascontiguousarray(v.transpose(2, 1, 0))).cuda()
    kt = torch.empty_like(vt)
    torch.cuda.synchronize()
    from cgd_b200.model import JacBands
    d.schur_solve_bands(kt, vt, JacBands(*Jt), 120.0)
    assert np.array_equal(kt.cpu().numpy().transpose(2, 1, 0), kg)
    assert np.array_equal(vt.cpu().numpy().transpose(2, 1, 0), vg)


def test_ten_steps(case):
    name, o, g, U, nu, d = case
    dt = 600.0 if name == "small" else 300.0
    Vo = o.ros_step(U, dt, 10)
    Vg = U.copy(order="F")
    d.time_stepper(Vg, dt, 10)
    assert np.all(np.isfinite(Vg))
    _same(Vg, Vo, d.exact, TOL_STEP)


def test_device_pointers_match_host(case):
    """Zero-copy device arrays (torch CUDA tensors) give the same result as
    host arrays staged through the library."""
    import torch
    name, o, g, U, nu, d = case
    Fh = d.fcn(U)
    Ut = torch.from_numpy(np.ascontiguousarray(U.transpose(2, 1, 0))).cuda()
    torch.cuda.synchronize()
    Ft = torch.empty_like(Ut)
    d.fcn(Ut, Ft)
    assert np.array_equal(Ft.cpu().numpy().transpose(2, 1, 0), Fh)
    Vh = U.copy(order="F")
    d.time_stepper(Vh, 300.0, 2)
    d.time_stepper(Ut, 300.0, 2)
    torch.cuda.synchronize()
    assert np.array_equal(Ut.cpu().numpy().transpose(2, 1, 0), Vh)


def test_deterministic(case):
    name, o, g, U, nu, d = case
    a = U.copy(order="F")
    b = U.copy(order="F")
    d.time_stepper(a, 300.0, 3)
    d.time_stepper(b, 300.0, 3)
    assert np.array_equal(a, b)


def test_mass_integral(case):
    name, o, g, U, nu, d = case
    m0 = d.mass_integral(U)
    assert abs(m0 - o.mass_integral(U)) <= 1e-14 * abs(m0)
    V = U.copy(order="F")
    d.time_stepper(V, 300.0, 5)
    assert abs(d.mass_integral(V) - m0) <= 1e-13 * abs(m0)


def test_nonfinite_state_reported(oracle_mod, lib_ready):
    """A NaN written into the state on the host is detected after the step and
    reported as CGD_ERR_NONFINITE (no device trap)."""
    from cgd_b200 import CgdError
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 0)
    d = _dycore(g, 0, nu, check_finite=True)
    V = U.copy(order="F")
    d.time_stepper(V, 300.0, 1)
    V[2, 5, 4] = np.nan
    with pytest.raises(CgdError) as e:
        d.time_stepper(V, 300.0, 1)
    assert e.value.code == -4
    d.close()


@pytest.mark.parametrize("variant", ["exact", "fast"])
def test_dropin_configuration(oracle_mod, lib_ready, variant):
    """nPanel 30, p 4, nz 45 quadratic, 2 tracers: the full-size drop-in case."""
    o, g, U, nu = make_case(oracle_mod, 30, 4, 45, 2, "quadratic")
    d = _dycore(g, 2, nu, exact=(variant == "exact"))
    _same(d.fcn(U), o.rhs(U), d.exact, TOL_RHS)
    Vo = o.ros_step(U, 120.0, 2)
    Vg = U.copy(order="F")
    d.time_stepper(Vg, 120.0, 2)
    _same(Vg, Vo, d.exact, TOL_STEP)
    d.close()


@pytest.mark.parametrize("variant", ["exact", "fast"])
def test_two_layers(oracle_mod, lib_ready, variant):
    """nz = 2, a single interface: tendency, Jacobian and Schur solve.  (The
    restated reference integration itself blows up within ten steps on two
    layers at any dt tried down to 10 s, so no steps are compared here.)"""
    o, g, U, nu = make_case(oracle_mod, 4, 4, 2, 1, "uniform")
    d = _dycore(g, 1, nu, exact=(variant == "exact"))
    _same(d.fcn(U), o.rhs(U), d.exact, TOL_RHS)
    bo, bg = o.jac(U), d.jac(U)
    assert np.abs(bg - bo).max() <= 1e-14 * np.abs(bo).max()
    v = np.asfortranarray(np.random.default_rng(3).standard_normal(U.shape))
    ko, vo = o.schur(v, 300.0)
    vg = v.copy(order="F")
    kg = d.schur_solve(vg, 300.0)
    _same(kg, ko, d.exact, TOL_RHS)
    _same(vg, vo, d.exact, TOL_RHS)
    d.close()
