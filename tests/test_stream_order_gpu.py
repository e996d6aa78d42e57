"""Calls wait for the work the caller queued on its own stream before they
read their arguments (cgd_set_caller_stream).  A bounded spin kernel on the
caller's stream holds back a copy into the state; a call that did not wait
would read the stale state.  Checked on the default (legacy) stream, which
PyTorch uses, and on a side stream named through set_caller_stream."""
import numpy as np
import pytest

from _cases import make_case

pytestmark = pytest.mark.gpu

SPIN_CYCLES = 50_000_000   # about 25 ms at 2 GHz


@pytest.fixture(scope="module")
def case(oracle_mod, built_lib, cuda_ok):
    import torch
    from cgd_b200 import Dycore
    o, g, U, nu = make_case(oracle_mod, 4, 4, 8, 0, "quadratic")
    d = Dycore(g, 0, nu)
    U = np.asfortranarray(U)
    Ut = torch.from_numpy(np.ascontiguousarray(U.transpose(2, 1, 0))).cuda()
    yield d, U, Ut, torch
    d.close()


def test_default_stream_work_is_waited_for(case):
    d, U, Ut, torch = case
    F_ref = d.fcn(U)
    Z = torch.zeros_like(Ut)
    torch.cuda.synchronize()
    torch.cuda._sleep(SPIN_CYCLES)
    Z.copy_(Ut)                       # queued behind the spin
    F = torch.empty_like(Ut)
    d.fcn(Z, F)
    assert np.array_equal(F.cpu().numpy().transpose(2, 1, 0), F_ref)


def test_side_stream_named_by_the_caller(case):
    d, U, Ut, torch = case
    V_ref = U.copy(order="F")
    d.time_stepper(V_ref, 300.0, 2)
    s = torch.cuda.Stream()
    Z = torch.zeros_like(Ut)
    torch.cuda.synchronize()
    d.set_caller_stream(s.cuda_stream)
    try:
        with torch.cuda.stream(s):
            torch.cuda._sleep(SPIN_CYCLES)
            Z.copy_(Ut)
        d.time_stepper(Z, 300.0, 2)
    finally:
        d.set_caller_stream(None)
    assert np.array_equal(Z.cpu().numpy().transpose(2, 1, 0), V_ref)
