"""The hand-written adjoint of the tendency (cgd_rhs_adjoint) against central
finite differences of the forward tendency on the GPU (dot-product test):

    <lambda, (F(U + eps v) - F(U - eps v)) / (2 eps)>  ==  <(dF/dU)^T lambda, v>

for every pair (output field of lambda, input field of v), at a state with
vertical motion (the initial state has w = 0, where the upwind flux sits on
the kink of |w|).  The difference is measured against sum |lambda * dF|; the
finite differences are accurate to about 1e-9 of that at eps = 1e-6."""
import numpy as np
import pytest

from _cases import make_case

pytestmark = pytest.mark.gpu

TOL = 1e-7


@pytest.mark.parametrize("case", [(4, 4, 8, "quadratic"), (3, 3, 6, "uniform"), (3, 2, 5, "quadratic")])
def test_tendency_adjoint_dot_products(oracle_mod, built_lib, cuda_ok, case):
    from cgd_b200 import Dycore
    n, p, nz, st = case
    o, g, U, nu = make_case(oracle_mod, n, p, nz, 0, st)
    d = Dycore(g, 0, nu, exact=True)
    U = np.asfortranarray(U)
    d.time_stepper(U, 300.0, 5)
    rng = np.random.default_rng(7)
    scale = np.array([max(np.abs(U[:, :, f]).max(), 1.0) for f in range(5)])
    eps = 1e-6
    worst = 0.0
    for fo in range(5):
        for fi in range(5):
            lam = np.zeros_like(U)
            lam[:, :, fo] = rng.standard_normal(U.shape[:2])
            lam = np.asfortranarray(lam)
            v = np.zeros_like(U)
            v[:, :, fi] = rng.standard_normal(U.shape[:2]) * scale[fi]
            dF = (d.fcn(np.asfortranarray(U + eps * v)) - d.fcn(np.asfortranarray(U - eps * v))) / (2 * eps)
            lhs = np.sum(lam * dF)
            rhs = np.sum(d.fcn_adjoint(U, lam) * v)
            err = abs(lhs - rhs) / (np.sum(np.abs(lam * dF)) + 1e-300)
            worst = max(worst, err)
            assert err <= TOL, (fo, fi, lhs, rhs, err)
    d.close()


def test_tendency_adjoint_rejects_tracers(oracle_mod, built_lib, cuda_ok):
    from cgd_b200 import CgdError, Dycore
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 1)
    d = Dycore(g, 1, nu)
    with pytest.raises(CgdError) as e:
        d.fcn_adjoint(U, np.asfortranarray(np.ones_like(U)))
    assert e.value.code == -7
    d.close()
