"""Analytic checks of the oracle itself (the reference pins no tendency,
Jacobian or step values, so these invariants back the CPU restatement):
mass conservation of the continuity tendency and of the Rosenbrock step,
a resting isothermal atmosphere staying nearly at rest, the Schur solve
inverting (I/fac - J), and first-order-in-dt consistency of the step."""
import numpy as np
import pytest

from cgd_b200 import grid as G
from cgd_b200 import physics as Ph


@pytest.fixture(scope="module")
def small(oracle_mod):
    cfg = Ph.CONFIGS["small"]
    z = cfg.levels()
    nu = Ph.hyperdiffusion(cfg.nPanel, cfg.OrdPoly)
    o = oracle_mod.Oracle(cfg.nPanel, cfg.OrdPoly, cfg.nz, 0, z, nu=nu, Up=1.0)
    U = o.init_state()
    Ph.theta_noise(U, 0.01, cfg.seed_theta)
    return o, U, cfg


def test_mass_conservation(small):
    o, U, cfg = small
    F = o.rhs(U)
    M, MM = o.mass()
    # lumped mass weighted continuity tendency sums to round-off
    tot = o.mass_integral(U)
    assert abs(o.mass_integral(F)) * cfg.dt < 1e-13 * tot
    V = o.ros_step(U, cfg.dt, 3)
    assert abs(o.mass_integral(V) - tot) < 1e-13 * tot


def test_initial_state_matches_product(small, oracle_mod):
    o, _, cfg = small
    g = G.init_grid_sphere(cfg.nPanel, cfg.OrdPoly, cfg.levels(), cfg.H, 6.371e6)
    Uo = o.init_state()
    Up = Ph.initial_state(g, Ph.PhysParameters(), 0, None, 1.0)
    for v in range(5):
        scale = max(np.abs(Uo[:, :, v]).max(), 1.0)
        assert np.abs(Up[:, :, v] - Uo[:, :, v]).max() <= 1e-12 * scale


def test_resting_isothermal_atmosphere(oracle_mod):
    """A hydrostatically balanced isothermal rest state (discretely balanced up
    to truncation) only drives small vertical accelerations."""
    cfg = Ph.CONFIGS["small"]
    z = cfg.levels()
    o = oracle_mod.Oracle(cfg.nPanel, cfg.OrdPoly, cfg.nz, 0, z, nu=(0, 0, 0))
    g = G.init_grid_sphere(cfg.nPanel, cfg.OrdPoly, z, cfg.H, 6.371e6)
    ph = Ph.PhysParameters()
    T0 = 250.0
    U = np.zeros((cfg.nz, o.NumG, 5), order="F")
    zm = 0.5 * (z[:-1] + z[1:])
    p = ph.p0 * np.exp(-ph.Grav * zm / (ph.Rd * T0))
    rho = p / (ph.Rd * T0)
    th = T0 * (ph.p0 / p) ** ph.kappa
    U[:, :, 0] = rho[:, None]
    U[:, :, 4] = (rho * th)[:, None]
    F = o.rhs(U)
    assert np.abs(F[:, :, 1]).max() < 1e-9 and np.abs(F[:, :, 2]).max() < 1e-9
    assert np.abs(F[:, :, 0]).max() < 1e-12
    assert np.abs(F[:, :, 3]).max() < 0.05 * ph.Grav


def test_schur_inverts_operator(small):
    o, U, cfg = small
    bands = o.jac(U)
    rng = np.random.default_rng(3)
    v = np.asfortranarray(rng.standard_normal(U.shape))
    v[-1, :, 3] = 0.0
    fac = 300.0
    k, _ = o.schur(v.copy(order="F"), fac)
    # apply (I/fac - J) to k and compare with v
    JRhoW, JWRho, JWRhoTh, JRhoThW = bands
    nz = U.shape[0]
    r = k / fac
    kw = k[:-1, :, 3]
    # rho, rho*theta rows: - JRhoW w, - JRhoThW w (lower bidiagonal)
    for f, B in ((0, JRhoW), (4, JRhoThW)):
        r[:-1, :, f] -= B[0] * kw
        r[1:, :, f] -= B[1] * kw
    # w rows: - JWRho rho - JWRhoTh rhotheta (upper bidiagonal)
    r[:-1, :, 3] -= JWRho[1] * k[:-1, :, 0] + JWRho[0] * k[1:, :, 0]
    r[:-1, :, 3] -= JWRhoTh[1] * k[:-1, :, 4] + JWRhoTh[0] * k[1:, :, 4]
    r[-1, :, 3] = 0.0
    err = np.abs(r - v).max() / np.abs(v).max()
    assert err < 1e-10
