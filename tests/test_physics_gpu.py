"""Column physics of the tendency tail (cgd_set_physics): the dry
Held-Suarez forcing and the Rayleigh damping of w near the top, against the
oracle's restatement of ForceKernel!/DampKernel!.  The exact build is
bit-identical, the fast build within the FP64 bars; the adjoints refuse a
handle with physics; switching the terms off restores the plain tendency."""
import numpy as np
import pytest

from _cases import make_case, rel_err_per_field

pytestmark = pytest.mark.gpu

DAMP = (30000.0, 10000.0, 1.0 / 3600.0)


def _hs_vector():
    from cgd_b200.physics import HELD_SUAREZ, HELD_SUAREZ_ORDER
    return [HELD_SUAREZ[k] for k in HELD_SUAREZ_ORDER]


@pytest.mark.parametrize("variant", ["exact", "fast"])
@pytest.mark.parametrize("case", [(4, 4, 10, 0, "uniform"), (5, 3, 12, 2, "quadratic")])
def test_physics_matches_oracle(oracle_mod, built_lib, cuda_ok, variant, case):
    from cgd_b200 import Dycore
    n, p, nz, NT, st = case
    o, g, U, nu = make_case(oracle_mod, n, p, nz, NT, st)
    exact = variant == "exact"
    d = Dycore(g, NT, nu, exact=exact)
    F0 = d.fcn(U)
    o.set_physics(_hs_vector(), DAMP)
    d.set_physics(True, DAMP)
    Fo, Fg = o.rhs(U), d.fcn(U)
    assert not np.array_equal(Fo, F0)   # the terms act
    err = rel_err_per_field(Fg, Fo)
    assert err.max() <= 1e-12, err
    if exact:
        assert np.array_equal(Fg, Fo)
    Vo = o.ros_step(U, 300.0, 5)
    Vg = U.copy(order="F")
    d.time_stepper(Vg, 300.0, 5)
    err = rel_err_per_field(Vg, Vo)
    assert err.max() <= 1e-10, err
    if exact:
        assert np.array_equal(Vg, Vo)
    # off again: the plain tendency
    d.set_physics(None, None)
    assert np.array_equal(d.fcn(U), F0)
    d.close()


def test_adjoint_refuses_physics(oracle_mod, built_lib, cuda_ok):
    from cgd_b200 import CgdError, Dycore
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 0)
    d = Dycore(g, 0, nu)
    d.set_physics(True, None)
    with pytest.raises(CgdError) as e:
        d.fcn_adjoint(U, U)
    assert e.value.code == -7
    d.close()
