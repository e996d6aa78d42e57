"""The owner gather (DSS) for global DOFs with more than four contributors.

A cubed-sphere node has one to four contributors, and the gather reads the
first four from one row of a per-DOF table; a grid with more (any Glob the
caller passes to cgd_create) takes the general path over the contributor
list.  Merging DOF B into DOF A of a small grid makes such a DOF: five
contributors (A with four, B with one) or eight (two with four).  The
oracle's element-node contributions of the merged grid are those of the
original grid with B's column and mass set to A's, summed here in ascending
(element, node) order like the library's gather."""
import numpy as np
import pytest

from _cases import make_case, merge_dofs, ordered_dss, rel_err_per_field


def _pick(g, ca, cb):
    cnt = np.bincount(np.asarray(g.glob).ravel() - 1, minlength=g.NumG)
    a = np.nonzero(cnt == ca)[0]
    b = np.nonzero(cnt == cb)[0]
    A = int(a[len(a) // 3])
    B = int([x for x in b if x != A][len(b) // 2])
    return A, B


def test_ordered_dss_is_the_oracle_phase1_cache(oracle_mod):
    """The summation order used below reproduces the oracle's own DSS, of
    the phase-1 cache and of the tendency."""
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 1, "quadratic")
    T1 = ordered_dss(o.contributions(U), g.glob, g.NumG)
    assert np.array_equal(T1, o.hypervisc1(U))
    assert np.array_equal(ordered_dss(o.contributions(U, T1), g.glob, g.NumG), o.rhs(U))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["exact", "fast"])
@pytest.mark.parametrize("counts", [(4, 1), (4, 4)], ids=["five", "eight"])
def test_phase1_gather_with_many_contributors(oracle_mod, built_lib, cuda_ok, variant, counts):
    from cgd_b200 import Dycore
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 1, "quadratic")
    A, B = _pick(g, *counts)
    g2, U2, Uo = merge_dofs(o, g, U, A, B)
    cnt2 = np.bincount(np.asarray(g2.glob).ravel() - 1, minlength=g2.NumG)
    assert cnt2.max() == sum(counts)
    want = ordered_dss(o.contributions(Uo), g2.glob, g2.NumG)
    d = Dycore(g2, 1, nu, exact=(variant == "exact"))
    try:
        got = d.hypervisc_phase1(U2)
        F = d.fcn(U2)
    finally:
        d.close()
    err = rel_err_per_field(got, want)
    if variant == "exact":
        assert np.array_equal(got, want), err
    else:
        assert err.max() <= 1e-11, err
    # the tendency: phase 2 at the merged cache (B's nodes read A's), then
    # the same ordered gather (w: upper plus lower node of every contributor)
    old = np.arange(g.NumG)
    new = old - (old > B)
    new[B] = A - (A > B)
    Fw = ordered_dss(o.contributions(Uo, want[:, new, :]), g2.glob, g2.NumG)
    err = rel_err_per_field(F, Fw)
    if variant == "exact":
        assert np.array_equal(F, Fw), err
    else:
        assert err.max() <= 1e-12, err
