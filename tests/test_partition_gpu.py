"""Decomposed grid on the GPU: the parts of a 2- and 3-rank element partition
run together in one process (PartGroup: the same pack, exchange and unpack
of contributions as between processes, the transport being device copies)
and must reproduce the single-process tendency and Rosenbrock-W steps bit
for bit on every rank's DOFs - the contributors of a DOF are summed in the
same order whichever rank owns them.  The exact build is also compared with
the oracle."""
import numpy as np
import pytest

from _cases import make_case

pytestmark = pytest.mark.gpu


def _dev(U):
    import torch
    return torch.from_numpy(np.ascontiguousarray(U.transpose(2, 1, 0))).cuda()


def _host(t):
    return t.cpu().numpy().transpose(2, 1, 0)


@pytest.mark.parametrize("nranks", [2, 3])
@pytest.mark.parametrize("variant", ["exact", "fast"])
def test_group_matches_single_process(oracle_mod, built_lib, cuda_ok, nranks, variant):
    import torch
    from cgd_b200 import Dycore, PartGroup
    from cgd_b200.parallel import build_plans, partition_elements
    exact = variant == "exact"
    o, g, U, nu = make_case(oracle_mod, 4, 4, 12, 1, "quadratic")
    whole = Dycore(g, 1, nu, exact=exact)
    plans = build_plans(g, partition_elements(g.NF, nranks))
    parts = [Dycore(P.local_grid(g), 1, nu, exact=exact, halo=P) for P in plans]
    grp = PartGroup(parts)
    # tendency
    F1 = whole.fcn(U)
    Ul = [_dev(P.restrict(U)) for P in plans]
    Fl = [torch.empty_like(u) for u in Ul]
    grp.fcn(Ul, Fl)
    for P, f in zip(plans, Fl):
        assert np.array_equal(_host(f), F1[:, P.dofs, :])
    if exact:
        assert np.array_equal(F1, o.rhs(U))
    # steps
    V = U.copy(order="F")
    whole.time_stepper(V, 300.0, 3)
    grp.time_stepper(Ul, 300.0, 3)
    for P, u in zip(plans, Ul):
        assert np.array_equal(_host(u), V[:, P.dofs, :])
    if exact:
        assert np.array_equal(V, o.ros_step(U, 300.0, 3))
    # the global mass integral: each DOF counted on its owning rank
    m = sum(p.mass_integral(_host(u).copy(order="F")) for p, u in zip(parts, Ul))
    assert abs(m - whole.mass_integral(V)) <= 1e-13 * abs(m)
    for p in parts:
        p.close()
    whole.close()


def test_decomposed_grid_rejects_mixed_form(oracle_mod, built_lib, cuda_ok):
    from cgd_b200 import CgdError, Dycore
    from cgd_b200.parallel import build_plans, partition_elements
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 0)
    P = build_plans(g, partition_elements(g.NF, 2))[0]
    with pytest.raises(CgdError) as e:
        Dycore(P.local_grid(g), 0, nu, precision="mixed", halo=P)
    assert e.value.code == -7
