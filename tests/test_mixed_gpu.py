"""The mixed form (CGD_PREC_MIXED) on the GPU: horizontal derivative sums in
FP32 on perturbations from an FP64 per-level reference profile, everything
else in FP64.  Checked against the FP64 oracle and the FP64 GPU path:

  * tendencies within 5e-4 relative max-norm per field (u and v are small
    residuals of the balanced pressure-gradient and Coriolis terms, so their
    relative error is the largest: about 1e-4 measured);
  * 10 Rosenbrock-W steps within 1e-4 of the FP64 state per field;
  * mass conserved to 1e-11 relative over those steps.
"""
import numpy as np
import pytest

from _cases import make_case, rel_err_per_field

pytestmark = pytest.mark.gpu

CASES = {
    "p4": dict(nPanel=6, p=4, nz=10, NumTr=0, stretch="uniform"),
    "p3_tracers": dict(nPanel=5, p=3, nz=12, NumTr=2, stretch="quadratic"),
    "p4_nz30": dict(nPanel=8, p=4, nz=30, NumTr=1, stretch="quadratic"),
    # the mixed form's own configuration, reduced horizontally: p 4, nz 64
    # stretched quadratically, no tracers (nPanel 60 in the benchmark)
    "cfg3_shape": dict(nPanel=6, p=4, nz=64, NumTr=0, stretch="quadratic"),
}


@pytest.fixture(scope="module", params=list(CASES))
def pair(request, oracle_mod, built_lib, cuda_ok):
    from cgd_b200 import Dycore
    c = CASES[request.param]
    o, g, U, nu = make_case(oracle_mod, c["nPanel"], c["p"], c["nz"], c["NumTr"], c["stretch"])
    d64 = Dycore(g, c["NumTr"], nu)
    dm = Dycore(g, c["NumTr"], nu, precision="mixed")
    yield o, U, d64, dm
    d64.close()
    dm.close()


def test_mixed_tendency_close_to_oracle(pair):
    o, U, d64, dm = pair
    err = rel_err_per_field(dm.fcn(U), o.rhs(U))
    assert err.max() <= 5e-4, err


def test_mixed_steps_close_to_fp64(pair):
    o, U, d64, dm = pair
    V64 = U.copy(order="F")
    Vm = U.copy(order="F")
    d64.time_stepper(V64, 300.0, 10)
    dm.time_stepper(Vm, 300.0, 10)
    assert np.all(np.isfinite(Vm))
    err = rel_err_per_field(Vm, V64)
    assert err.max() <= 1e-4, err


def test_mixed_mass_conservation(pair):
    o, U, d64, dm = pair
    m0 = dm.mass_integral(U)
    V = U.copy(order="F")
    dm.time_stepper(V, 300.0, 10)
    assert abs(dm.mass_integral(V) - m0) <= 1e-11 * abs(m0)


def test_mixed_is_deterministic(pair):
    o, U, d64, dm = pair
    a = U.copy(order="F")
    b = U.copy(order="F")
    dm.time_stepper(a, 300.0, 3)
    dm.time_stepper(b, 300.0, 3)
    assert np.array_equal(a, b)
