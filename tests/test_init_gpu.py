"""The grid set-up on the GPU (cgd_metric_sphere, cgd_mass_dz, cgd_create
from device arrays) against the host set-up (grid.py, itself bit-equal to
the oracle):

  * the device metric agrees with the host metric to rounding (the device's
    sin/cos/asin/atan2 may differ from the host libm in the last bit);
  * the device mass and dz of the host metric are the host's bit for bit
    (same contributors, same order);
  * cgd_create from device copies of the host arrays forms the same element
    metric as from the host arrays: tendencies and steps bit for bit (exact
    build);
  * a Dycore on the device-built grid steps like the host-built one to
    rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(6, 4, 10, "uniform"), (4, 3, 12, "quadratic"), (3, 2, 7, "quadratic")]


def _levels(nz, stretch):
    from cgd_b200 import grid as G
    return G.vertical_uniform(nz, 30000.0) if stretch == "uniform" else G.vertical_quadratic(nz, 30000.0)


def _host(t, shape):
    """A CUDA tensor holding a Fortran-ordered array -> the numpy array."""
    return np.asfortranarray(t.cpu().numpy().reshape(-1).reshape(shape, order="F"))


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).transpose(*reversed(range(a.ndim))))).cuda()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("case", CASES)
def test_device_metric_and_mass(built_lib, cuda_ok, case):
    from cgd_b200 import _lib
    from cgd_b200 import grid as G
    n, p, nz, st = case
    z = _levels(nz, st)
    gh = G.init_grid_sphere(n, p, z, 30000.0, 6.371e6)
    gd = G.init_grid_sphere_device(n, p, z, 30000.0, 6.371e6)
    assert np.array_equal(gd.glob, gh.glob)
    for name in ("X", "dXdxI", "J"):
        a = _host(getattr(gd, name), getattr(gh, name).shape)
        assert _rel(a, getattr(gh, name)) <= 1e-13, name
    for name in ("M", "MMass", "dz"):
        a = _host(getattr(gd, name), getattr(gh, name).shape)
        assert _rel(a, getattr(gh, name)) <= 1e-13, name
    # the device mass and dz of the host metric: bit for bit
    import torch
    Jd, Xd = _dev(gh.J), _dev(gh.X)
    M = torch.empty_like(_dev(gh.M))
    MM = torch.empty_like(_dev(gh.MMass))
    dz = torch.empty_like(MM)
    g64 = np.asfortranarray(gh.glob, dtype=np.int64)
    w = np.ascontiguousarray(gh.w)
    _lib.check(_lib.lib().cgd_mass_dz(p, nz, gh.NF, gh.NumG, g64.ctypes.data, w.ctypes.data, Jd.data_ptr(),
                                      Xd.data_ptr(), M.data_ptr(), MM.data_ptr(), dz.data_ptr()), "cgd_mass_dz")
    assert np.array_equal(_host(M, gh.M.shape), gh.M)
    assert np.array_equal(_host(MM, gh.MMass.shape), gh.MMass)
    assert np.array_equal(_host(dz, gh.dz.shape), gh.dz)


@pytest.mark.parametrize("variant", ["exact", "fast"])
def test_create_from_device_arrays(oracle_mod, built_lib, cuda_ok, variant):
    """Device copies of the oracle's arrays give the same handle as the host
    arrays (the element metric compacted on the device)."""
    import dataclasses

    from _cases import make_case
    from cgd_b200 import Dycore
    o, g, U, nu = make_case(oracle_mod, 4, 4, 9, 1, "quadratic")
    exact = variant == "exact"
    dh = Dycore(g, 1, nu, exact=exact)
    gd = dataclasses.replace(g, X=_dev(g.X), dXdxI=_dev(g.dXdxI), J=_dev(g.J), M=_dev(g.M), dz=_dev(g.dz))
    dd = Dycore(gd, 1, nu, exact=exact)
    assert np.array_equal(dd.fcn(U), dh.fcn(U))
    a, b = U.copy(order="F"), U.copy(order="F")
    dh.time_stepper(a, 300.0, 3)
    dd.time_stepper(b, 300.0, 3)
    assert np.array_equal(a, b)
    if exact:
        assert np.array_equal(a, o.ros_step(U, 300.0, 3))
    dh.close()
    dd.close()


def test_device_grid_run_matches_host_grid(built_lib, cuda_ok):
    import dataclasses

    from cgd_b200 import physics as Ph
    from cgd_b200 import setup
    cfg = dataclasses.replace(Ph.CONFIGS["small"], nPanel=6, nz=10)
    dh, Uh, _ = setup(cfg)
    dd, Ud, _ = setup(cfg, where="device")
    assert np.abs(Ud - Uh).max() <= 1e-12 * np.abs(Uh).max()    # the initial state from the device X
    a, b = Uh.copy(order="F"), Uh.copy(order="F")
    dh.time_stepper(a, cfg.dt, 5)
    dd.time_stepper(b, cfg.dt, 5)
    for f in range(a.shape[2]):
        den = max(np.abs(a[..., f]).max(), 1e-300)
        assert np.abs(a[..., f] - b[..., f]).max() / den <= 1e-9, f
    dh.close()
    dd.close()
