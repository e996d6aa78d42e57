"""The hand-written adjoints of the tendency (cgd_rhs_adjoint) and of one
Rosenbrock-W step (cgd_ros_step_adjoint) against central finite differences
of the forward maps on the GPU (dot-product test, shown for the tendency):

    <lambda, (F(U + eps v) - F(U - eps v)) / (2 eps)>  ==  <(dF/dU)^T lambda, v>

for every pair (output field of lambda, input field of v), at a state with
vertical motion (the initial state has w = 0, where the upwind flux sits on
the kink of |w|).  The difference is measured against sum |lambda * dF|; the
finite differences are accurate to about 1e-9 of that at eps = 1e-6.

The step adjoint adds the transposed column Schur solve, the derivative of
the Jacobian bands with respect to the state and the stage combinations.  A
step perturbs w through the implicit solve, and the limited upwind flux is
piecewise linear in the reconstruction ratios: a dense perturbation of all
nodes crosses some of the limiter's kinks at any eps that rounding allows.
The step is therefore checked entry by entry: <lambda, dU1/dU0(l, g, f)>
from central differences of one perturbed entry, against the entry of
(dU1/dU0)^T lambda, at eps = 1e-5 ... 1e-8 of the field's scale (the
difference of the two perturbed runs is taken entry by entry before it is
weighted and summed); the best must agree to 1e-6.  With one entry
perturbed the nearest kink is usually farther away than that; an entry
whose differences disagree among themselves by more than 1e-6 (the map is
not smooth there at these scales) may be set aside, at most one in ten.  An entry whose
differences agree with each other but not with the adjoint always fails.
Chained over checkpoints, the same check is made for the gradient of a
functional of the state after several steps."""
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


@pytest.mark.parametrize("case", [(4, 4, 8, "quadratic"), (3, 3, 6, "uniform")])
def test_tendency_adjoint_against_oracle_directional_derivatives(oracle_mod, built_lib, cuda_ok, case):
    """The GPU tendency adjoint against FP64 directional derivatives of the
    CPU restatement's tendency (central differences of the oracle's RHS):
    <lambda, dF_oracle(U; v)> == <(dF/dU)^T lambda, v> for dense random
    lambda and v over all fields."""
    from cgd_b200 import Dycore
    n, p, nz, st = case
    o, g, U, nu = make_case(oracle_mod, n, p, nz, 0, st)
    d = Dycore(g, 0, nu, exact=True)
    U = np.asfortranarray(U)
    d.time_stepper(U, 300.0, 5)
    rng = np.random.default_rng(20261205)
    scale = np.array([max(np.abs(U[:, :, f]).max(), 1.0) for f in range(5)])
    eps = 1e-6
    for _ in range(4):
        lam = np.asfortranarray(rng.standard_normal(U.shape))
        v = np.asfortranarray(rng.standard_normal(U.shape) * scale)
        dF = (o.rhs(np.asfortranarray(U + eps * v)) - o.rhs(np.asfortranarray(U - eps * v))) / (2 * eps)
        lhs = np.sum(lam * dF)
        rhs = np.sum(d.fcn_adjoint(U, lam) * v)
        err = abs(lhs - rhs) / (np.sum(np.abs(lam * dF)) + 1e-300)
        assert err <= TOL, (lhs, rhs, err)
    d.close()


def test_tendency_adjoint_rejects_tracers(oracle_mod, built_lib, cuda_ok):
    from cgd_b200 import CgdError, Dycore
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 1)
    d = Dycore(g, 1, nu)
    with pytest.raises(CgdError) as e:
        d.fcn_adjoint(U, np.asfortranarray(np.ones_like(U)))
    assert e.value.code == -7
    d.close()


def _evolved(oracle_mod, case, NumTr=0):
    from cgd_b200 import Dycore
    n, p, nz, st = case
    o, g, U, nu = make_case(oracle_mod, n, p, nz, NumTr, st)
    d = Dycore(g, NumTr, nu, exact=True)
    U = np.asfortranarray(U)
    d.time_stepper(U, 300.0, 5)
    scale = np.array([max(np.abs(U[:, :, f]).max(), 1.0) for f in range(U.shape[2])])
    return d, U, scale


def _step(d, U, dt, n):
    V = np.array(U, order="F", copy=True)
    d.time_stepper(V, dt, n)
    return V


def _entry_check(U, scale, Gdiff, adj, nodes, rels=(1e-5, 1e-6, 1e-7, 1e-8), tol=1e-6):
    """Compare adj[l, g, f] with central differences G(U + h e) - G(U - h e)
    = Gdiff(U + h e, U - h e) of a scalar map G along the unit entry
    e = (l, g, f), at the step sizes rels (of the field's scale).  Returns the entries that fail (smooth
    but different) and those set aside (not smooth)."""
    failed, aside = [], []
    for (l, gg, f) in nodes:
        den = max(abs(adj[l, gg, f]), np.median(np.abs(adj[:, :, f])) + 1e-300)
        fds = []
        for eps in rels:
            h = eps * scale[f]
            Up = U.copy(order="F")
            Up[l, gg, f] += h
            Um = U.copy(order="F")
            Um[l, gg, f] -= h
            fds.append(Gdiff(Up, Um) / (2 * h))
        err = min(abs(x - adj[l, gg, f]) for x in fds) / den
        spread = (max(fds) - min(fds)) / den
        if err > tol:
            (aside if spread > tol else failed).append(((l, gg, f), adj[l, gg, f], fds, err))
    return failed, aside


def _assert_entries(failed, aside, nodes):
    assert not failed, failed
    assert len(aside) <= len(nodes) // 10, aside


def _nodes(rng, shape, per_field):
    nz, NumG, NV = shape
    return [(int(i % nz), int(rng.integers(NumG)), f) for f in range(NV) for i in range(per_field)]


@pytest.mark.parametrize("case,dt", [((4, 4, 8, "quadratic"), 300.0), ((4, 4, 8, "quadratic"), 30.0),
                                     ((3, 3, 6, "uniform"), 300.0)])
def test_step_adjoint_entries(oracle_mod, built_lib, cuda_ok, case, dt):
    d, U, scale = _evolved(oracle_mod, case)
    rng = np.random.default_rng(11)
    lam = np.asfortranarray(rng.standard_normal(U.shape))
    U0 = U.copy(order="F")
    Lin = d.ros_step_adjoint(U, lam, dt)
    assert np.array_equal(U, U0)
    nodes = _nodes(rng, U.shape, 2 * U.shape[0])
    _assert_entries(*_entry_check(U, scale, lambda A, B: np.sum(lam * (_step(d, A, dt, 1) - _step(d, B, dt, 1))), Lin, nodes), nodes)
    d.close()


def test_checkpointed_gradient_of_a_functional(oracle_mod, built_lib, cuda_ok):
    """J(U0) = 1/2 sum over a box of (rho theta)_n^2 after 5 steps; its
    gradient by the checkpointed chain of step adjoints (a checkpoint every 2
    steps, so segments are recomputed), entry by entry against central
    differences: the entries of largest gradient in every field and random
    ones."""
    d, U, scale = _evolved(oracle_mod, (3, 3, 6, "quadratic"))
    dt, n = 300.0, 5
    nz, NumG, NV = U.shape
    w = np.zeros(U.shape)
    w[1:4, : NumG // 3, 4] = 1.0 / scale[4]

    def Jdiff(A, B):
        a, b = _step(d, A, dt, n), _step(d, B, dt, n)
        return 0.5 * np.sum(w * (a - b) * (a + b))

    Un = _step(d, U, dt, n)
    grad = d.steps_adjoint(U, np.asfortranarray(w * Un), dt, n, every=2)
    # the same gradient without recomputation (every step kept) and with
    # replayed instead of recorded steps; the adjoint sums are atomic, so
    # they agree to rounding
    g1 = d.steps_adjoint(U, np.asfortranarray(w * Un), dt, n, every=1)
    assert np.abs(grad - g1).max() <= 1e-10 * np.abs(g1).max()
    g2 = d.steps_adjoint(U, np.asfortranarray(w * Un), dt, n, every=2, tape=False)
    assert np.abs(grad - g2).max() <= 1e-10 * np.abs(g2).max()
    rng = np.random.default_rng(5)
    nodes = []
    for f in range(NV):
        top = np.argsort(np.abs(grad[:, :, f]).ravel(order="F"))[-3:]
        nodes += [(int(i % nz), int(i // nz), f) for i in top]
    nodes += _nodes(rng, U.shape, 2)
    _assert_entries(*_entry_check(U, scale, Jdiff, grad, nodes), nodes)
    d.close()


def test_box_pressure_functional_gradient(oracle_mod, built_lib, cuda_ok):
    """The adjoint workload's functional (mean squared lowest-layer pressure
    anomaly over a latitude/longitude box) on a small grid: its gradient
    after 4 steps with a checkpoint every 2, entry by entry against central
    differences, at the entries of largest gradient in every field and at
    random ones.  (Over longer windows and wider boxes the perturbation of
    one entry reaches enough limiter kinks that central differences stop
    being a 1e-6 reference; the chain itself is the same.)"""
    from cgd_b200.adjoint import BoxPressureFunctional, box_columns
    d, U, scale = _evolved(oracle_mod, (3, 3, 6, "quadratic"))
    box = box_columns(d.grid, (30.0, 60.0), (30.0, 90.0))
    assert box.size > 0
    Jf = BoxPressureFunctional(d, 300.0, 4, box=box, every=2)
    J, G = Jf.value_and_grad(U)
    assert J > 0 and np.all(np.isfinite(G))
    nz, NumG, NV = U.shape
    rng = np.random.default_rng(20261205)
    nodes = []
    for f in range(NV):
        a = np.abs(G[:, :, f]).ravel(order="F")
        top = np.argsort(a)[-3:]
        # random entries among those with at least 1 % of the field's largest
        # sensitivity (below that, the change of J is at its rounding level)
        sig = np.nonzero(a >= 1e-2 * a.max())[0]
        pick = rng.choice(sig, size=min(2, sig.size), replace=False)
        nodes += [(int(i % nz), int(i // nz), f) for i in np.concatenate([top, pick])]
    # J is a small change of p1 ~ 1e5 Pa: rounding of the perturbed runs
    # limits central differences to about 1e-6 of the entry (larger steps
    # meet the limiter's kinks), so this check of the functional's seed and
    # its direct term uses 1e-5
    _assert_entries(*_entry_check(U, scale, Jf.diff, G, nodes, rels=(1e-3, 1e-4, 1e-5, 1e-6), tol=1e-5),
                    nodes)
    d.close()


def test_recorded_step_matches_replayed_step(oracle_mod, built_lib, cuda_ok):
    """cgd_tape_record_step advances the state exactly as cgd_ros_step does,
    and the adjoint read from its record equals cgd_ros_step_adjoint's."""
    d, U, scale = _evolved(oracle_mod, (3, 3, 6, "quadratic"))
    rng = np.random.default_rng(3)
    lam = np.asfortranarray(rng.standard_normal(U.shape))
    V = U.copy(order="F")
    d.tape_record_step(0, V, 300.0)
    assert np.array_equal(V, _step(d, U, 300.0, 1))
    a = d.tape_step_adjoint(0, lam)
    b = d.ros_step_adjoint(U, lam, 300.0)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    d.tape_release()
    from cgd_b200 import CgdError
    with pytest.raises(CgdError):
        d.tape_step_adjoint(0, lam)
    d.close()


def test_step_adjoint_rejects_mixed(oracle_mod, built_lib, cuda_ok):
    from cgd_b200 import CgdError, Dycore
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 0)
    d = Dycore(g, 0, nu, precision="mixed")
    with pytest.raises(CgdError) as e:
        d.ros_step_adjoint(U, np.asfortranarray(np.ones_like(U)), 300.0)
    assert e.value.code == -7
    d.close()
