"""Batched ensemble on the GPU: members on different grids (nPanel, nz) and
with different dt advance together through cgd_batch_step, one graph per
ensemble step: 15 launches (split form), one persistent cooperative launch
per stage (fused form), or one graph branch per member running that
member's own step (members form).  All forms run the single-member kernel
bodies on the same data in the same order, so every member must come out
bit-identical to stepping it on its own, in every form and with or without
the autotuner."""
import numpy as np
import pytest

from _cases import make_case

pytestmark = pytest.mark.gpu

MEMBERS = [(4, 4, 10, "uniform", 600.0), (5, 4, 16, "quadratic", 300.0), (3, 4, 30, "quadratic", 300.0)]


def _members(oracle_mod, exact, precision="fp64"):
    from cgd_b200 import Dycore
    out = []
    for i, (n, p, nz, st, dt) in enumerate(MEMBERS):
        o, g, U, nu = make_case(oracle_mod, n, p, nz, 0, st, noise=0.01 + 0.01 * i)
        out.append((Dycore(g, 0, nu, exact=exact, precision=precision), U, dt))
    return out


def _dev(U):
    import torch
    return torch.from_numpy(np.ascontiguousarray(U.transpose(2, 1, 0))).cuda()


def _host(t):
    return t.cpu().numpy().transpose(2, 1, 0)


@pytest.mark.parametrize("exact,autotune,precision,form", [
    (True, False, "fp64", "split"), (False, True, "fp64", "split"), (False, False, "mixed", "split"),
    (True, False, "fp64", "fused"), (False, False, "fp64", "fused"), (False, False, "mixed", "fused"),
    (True, False, "fp64", "members"), (False, False, "mixed", "members")])
def test_batch_matches_members(oracle_mod, built_lib, cuda_ok, exact, autotune, precision, form):
    import torch
    from cgd_b200 import Ensemble
    mem = _members(oracle_mod, exact, precision)
    ref = []
    for d, U, dt in mem:
        V = _dev(U)
        d.time_stepper(V, dt, 3)
        torch.cuda.synchronize()
        ref.append(_host(V))
    # fresh handles for the batch (a mixed handle keeps the reference profile
    # of its first state, the same here)
    mem2 = _members(oracle_mod, exact, precision)
    ens = Ensemble([d for d, _, _ in mem2], autotune=autotune, fused=form == "fused",
                   members_form=form == "members")
    states = [_dev(U) for _, U, _ in mem2]
    ens.step(states, [dt for _, _, dt in mem2], 2)
    # the last step on copies: new state pointers (the members form captures
    # its graph again)
    states = [s.clone() for s in states]
    ens.step(states, [dt for _, _, dt in mem2], 1)
    torch.cuda.synchronize()
    for r, s in zip(ref, states):
        assert np.array_equal(_host(s), r)
    desc = ens.tuning()
    assert desc.startswith("order=")
    assert f"stage={form}" in desc or autotune
    if autotune:   # three orders x split, split with 8-level phase-2 CTAs, fused (OrdPoly 4), members
        assert desc.count("ms") == 12, desc
        assert "phase2_levels=" in desc
    ens.close()
    for d, _, _ in mem + mem2:
        d.close()


def test_batch_rejects_mismatched_members(oracle_mod, built_lib, cuda_ok):
    from cgd_b200 import CgdError, Dycore, Ensemble
    o, g, U, nu = make_case(oracle_mod, 3, 4, 6, 0)
    o2, g2, U2, nu2 = make_case(oracle_mod, 3, 3, 6, 0)
    a, b = Dycore(g, 0, nu), Dycore(g2, 0, nu2)
    with pytest.raises(CgdError) as e:
        Ensemble([a, b])
    assert e.value.code == -2
    a.close()
    b.close()


def test_batch_fused_needs_p4(oracle_mod, built_lib, cuda_ok):
    from cgd_b200 import CgdError, Dycore, Ensemble
    o, g, U, nu = make_case(oracle_mod, 3, 3, 6, 0)
    a = Dycore(g, 0, nu)
    with pytest.raises(CgdError) as e:
        Ensemble([a], fused=True)
    assert e.value.code == -7
    a.close()


def test_grid_barrier_holds_and_times_out(built_lib, cuda_ok):
    """The fused kernel's grid barrier: with every CTA present (two per SM,
    cooperative launch), no CTA passes any of 50 barriers before all have
    arrived; with a participant that never arrives, the wait ends after its
    0.2 s limit with CGD_ERR_TIMEOUT, and the device still runs a normal
    check afterwards."""
    import ctypes
    import time
    from cgd_b200 import _lib
    L = _lib.lib()
    v = ctypes.c_int32(-1)
    assert L.cgd_grid_barrier_check(50, 0, 2.0, ctypes.byref(v)) == 0
    assert v.value == 0
    t0 = time.perf_counter()
    assert L.cgd_grid_barrier_check(3, 1, 0.2, ctypes.byref(v)) == -5   # CGD_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    assert L.cgd_grid_barrier_check(50, 0, 2.0, ctypes.byref(v)) == 0
    assert v.value == 0
