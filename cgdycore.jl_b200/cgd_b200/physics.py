"""Physical parameters, the dry baroclinic-wave initial state and the run
configurations of the hot path.

* PhysParameters: src/DyCore/GlobalVariables.jl:188-230 (RadEarth is one
  parameter with the grid radius).
* BaroWaveExample: src/Examples/initial.jl:386-462 with
  ParamBaroWaveDrySphere (src/Examples/parameters.jl:48-83); the zonal-wind
  bump amplitude Up is a parameter (1 m/s here).
* InitialConditions: src/GPU/InitialConditions.jl:1-68 and the init kernels
  src/GPU/InitialKernel.jl:1-116 (values at layer midpoints, w at interface
  midpoints, the last element holding a node writes it).
"""
from dataclasses import dataclass, field

import numpy as np

PI = 3.141592653589793


@dataclass
class PhysParameters:
    RadEarth: float = 6.371e6
    Grav: float = 9.80616
    Cpd: float = 1004.0
    Cvd: float = 717.0
    p0: float = 1.0e5
    Omega: float = 2.0 * PI / 24.0 / 3600.0

    @property
    def Rd(self):
        return self.Cpd - self.Cvd

    @property
    def kappa(self):
        return self.Rd / self.Cpd


def barowave_profile(x, y, z, phys, Up=1.0):
    """(rho, u, v, w, theta) of the Ullrich et al. dry baroclinic wave at
    Cartesian points (vectorised)."""
    T0E, T0P, B, K, Lapse = 310.0, 240.0, 2.0, 3.0, 0.005
    PertExpR, PertLon, PertLat, PertZ = 0.1, PI / 9.0, 2.0 * PI / 9.0, 15000.0
    Rd, g = phys.Rd, phys.Grav
    r = np.sqrt(x * x + y * y + z * z)
    Lat = np.arcsin(z / r)
    Lon = np.arctan2(y, x)
    Lon = np.where(y < 0.0, Lon + 2.0 * PI, Lon)
    Z = np.maximum(r - phys.RadEarth, 0.0)
    T0 = 0.5 * (T0E + T0P)
    ConstA = 1.0 / Lapse
    ConstB = (T0 - T0P) / (T0 * T0P)
    ConstC = 0.5 * (K + 2.0) * (T0E - T0P) / (T0E * T0P)
    ConstH = Rd * T0 / g
    SZ = Z / (B * ConstH)
    Tau1 = ConstA * Lapse / T0 * np.exp(Lapse / T0 * Z) + ConstB * (1.0 - 2.0 * SZ * SZ) * np.exp(-SZ * SZ)
    Tau2 = ConstC * (1.0 - 2.0 * SZ * SZ) * np.exp(-SZ * SZ)
    IntTau1 = ConstA * (np.exp(Lapse / T0 * Z) - 1.0) + ConstB * Z * np.exp(-SZ * SZ)
    IntTau2 = ConstC * Z * np.exp(-SZ * SZ)
    cl = np.cos(Lat)
    Interior = cl ** K - K / (K + 2.0) * cl ** (K + 2.0)
    Temperature = 1.0 / (Tau1 - Tau2 * Interior)
    Pressure = phys.p0 * np.exp(-g / Rd * (IntTau1 - IntTau2 * Interior))
    Rho = Pressure / (Rd * Temperature)
    Th = Temperature * (phys.p0 / Pressure) ** (Rd / phys.Cpd)
    InteriorU = cl ** (K - 1.0) - cl ** (K + 1.0)
    BigU = g / phys.RadEarth * K * IntTau2 * InteriorU * Temperature
    RCosLat = phys.RadEarth * cl
    ORC = phys.Omega * RCosLat
    uS = -ORC + np.sqrt(ORC * ORC + RCosLat * BigU)
    GC = np.arccos(np.sin(PertLat) * np.sin(Lat) + np.cos(PertLat) * cl * np.cos(Lon - PertLon)) / PertExpR
    Taper = np.where(Z < PertZ, 1.0 - 3.0 * Z * Z / (PertZ * PertZ) + 2.0 * Z * Z * Z / (PertZ * PertZ * PertZ), 0.0)
    uS = uS + np.where(GC < 1.0, Up * Taper * np.exp(-GC * GC), 0.0)
    return Rho, uS, np.zeros_like(uS), np.zeros_like(uS), Th


def initial_state(grid, phys, NumTr=0, tracer_lonlat=None, Up=1.0):
    """U (nz, NumG, 5+NumTr), Fortran order: rho, u, v, w, rho*theta, rho*q."""
    from .grid import node_positions
    nz, numg = grid.nz, grid.NumG
    NV = 5 + NumTr
    U = np.zeros((nz, numg, NV), order="F")
    # the last element (highest index) holding a node writes it
    P = node_positions(grid)                                       # (numg, 2, 3, nz)
    mid = 0.5 * (P[:, 0] + P[:, 1])                                # (numg, 3, nz)
    xm, ym, zm = mid[:, 0, :], mid[:, 1, :], mid[:, 2, :]
    rho, u, v, _, th = barowave_profile(xm, ym, zm, phys, Up)
    U[:, :, 0] = rho.T
    U[:, :, 1] = u.T
    U[:, :, 2] = v.T
    U[:, :, 4] = (rho * th).T
    if nz > 1:
        xi = 0.5 * (P[:, 1, :, :-1] + P[:, 0, :, 1:])               # (numg, 3, nz-1)
        _, _, _, w, _ = barowave_profile(xi[:, 0], xi[:, 1], xi[:, 2], phys, Up)
        U[:-1, :, 3] = w.T
    if NumTr:
        r = np.sqrt(xm * xm + ym * ym + zm * zm)
        for iT in range(NumTr):
            lon, lat = tracer_lonlat[iT]
            c = (np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat))
            d = np.clip((xm * c[0] + ym * c[1] + zm * c[2]) / r, -1.0, 1.0)
            dist = phys.RadEarth * np.arccos(d) / 1.0e6
            U[:, :, 5 + iT] = (rho * np.exp(-dist * dist)).T
    return U


def theta_noise(U, amplitude, seed):
    """Add seeded uniform +-amplitude K theta noise at every column-level DOF
    (rho*theta += rho*dtheta); NumPy PCG64, column-major draw order."""
    nz, numg = U.shape[0], U.shape[1]
    rng = np.random.Generator(np.random.PCG64(seed))
    d = rng.uniform(-amplitude, amplitude, size=nz * numg).reshape((nz, numg), order="F")
    U[:, :, 4] += U[:, :, 0] * d
    return U


def member_perturbation(U, theta_amp, wind_amp, seed):
    """Seeded ensemble-member perturbation: uniform +-theta_amp K on theta
    (rho*theta += rho*dtheta) and +-wind_amp m/s on u and v at every
    column-level DOF; NumPy PCG64, column-major draw order (theta, u, v)."""
    nz, numg = U.shape[0], U.shape[1]
    rng = np.random.Generator(np.random.PCG64(seed))
    d = rng.uniform(-theta_amp, theta_amp, size=nz * numg).reshape((nz, numg), order="F")
    U[:, :, 4] += U[:, :, 0] * d
    U[:, :, 1] += rng.uniform(-wind_amp, wind_amp, size=nz * numg).reshape((nz, numg), order="F")
    U[:, :, 2] += rng.uniform(-wind_amp, wind_amp, size=nz * numg).reshape((nz, numg), order="F")
    return U


# Batched-ensemble workload: 48 members, 16 on each of three grids, seeded
# member perturbations (seed 20261300 + member), 6 simulated hours.  One dt
# for all members (108 s, 200 steps): it is below the explicit-acoustics
# limit of the finest member grid (nPanel 32; the limit scales with the grid
# spacing from the ~130 s of nPanel 30).
ENSEMBLE = {"grids": [(16, 30), (24, 45), (32, 64)], "per_grid": 16, "OrdPoly": 4, "dt": 108.0,
            "hours": 6.0, "theta_amp": 0.1, "wind_amp": 0.5, "seed0": 20261300}


# ParamHeldSuarezDrySphere (src/Examples/parameters.jl:122-131): the dry
# Held-Suarez forcing's rates (1/s) and equilibrium-temperature parameters.
_DAY = 3600.0 * 24.0
HELD_SUAREZ = {"k_a": 1.0 / (40.0 * _DAY), "k_f": 1.0 / _DAY, "k_s": 1.0 / (4.0 * _DAY), "DeltaT_y": 60.0,
               "DeltaTh_z": 10.0, "T_equator": 315.0, "T_min": 200.0, "sigma_b": 7.0 / 10.0}
HELD_SUAREZ_ORDER = ("k_a", "k_f", "k_s", "DeltaT_y", "DeltaTh_z", "T_equator", "T_min", "sigma_b")


def tracer_centres(NumTr, seed):
    """Blob centres uniform on the sphere: lon ~ U[0, 2pi), sin(lat) ~ U[-1, 1]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lon = rng.uniform(0.0, 2.0 * PI, size=NumTr)
    lat = np.arcsin(rng.uniform(-1.0, 1.0, size=NumTr))
    return np.stack([lon, lat], axis=1)


def hyperdiffusion(nPanel, OrdPoly):
    """nu = 5e14 (96/(n p))^2 for curl, grad and div (scaled with dx^2 from the
    reference's 5e14 at nPanel 32, p 3)."""
    nu = 5.0e14 * (96.0 / (nPanel * OrdPoly)) ** 2
    return nu, nu, nu


@dataclass
class RunConfig:
    name: str
    nPanel: int
    OrdPoly: int
    nz: int
    NumTr: int
    dt: float
    nsteps: int
    stretch: str           # "uniform" | "quadratic"
    H: float = 30000.0
    theta_noise: float = 0.01
    seed_theta: int = 20261203
    seed_tracer: int = 20261204
    Up: float = 1.0
    extra: dict = field(default_factory=dict)

    def levels(self):
        from . import grid as G
        if self.stretch == "uniform":
            return G.vertical_uniform(self.nz, self.H)
        return G.vertical_quadratic(self.nz, self.H)


# The adjoint workload's sensitivity study: J = mean squared lowest-layer
# pressure anomaly over the 10x10-degree box centred at 50N, 60E after 4 h
# (CONFIGS["adjoint"]: 120 steps of 120 s), gradient through the adjoint with
# a checkpoint every 8 steps, checked along seeded random directions.
ADJOINT_STUDY = {"box_lat": (45.0, 55.0), "box_lon": (55.0, 65.0), "every": 8, "fd_seed": 20261205, "fd_dirs": 8}

CONFIGS = {
    # small CPU-runnable case: 10 steps at dt 600 s
    "small": RunConfig("small", 6, 4, 10, 0, 600.0, 10, "uniform"),
    # the GPU drop-in grid: nPanel 30, p 4, nz 45 quadratic, 2 tracers, dt 120 s.
    # The horizontal acoustics of this W-method are explicit: at dt 300 s the run
    # blows up within 5 steps (max|w| 0.05 -> 8 m/s -> NaN), at 150 s within 40
    # steps; 120, 100 and 75 s stay stable for 600 steps (max|w| decays to
    # 3e-3 m/s).  1 day = 720 steps.
    "dropin": RunConfig("dropin", 30, 4, 45, 2, 120.0, 720, "quadratic",
                        extra={"dt_requested": 300.0}),
    # mixed-precision case: nPanel 60 halves the spacing; dt 60 s blows up within 60 steps, 50 s
    # (and 40 s) stays stable for a day: 1 day = 1728 steps
    "mixed": RunConfig("mixed", 60, 4, 64, 0, 50.0, 1728, "quadratic", extra={"dt_requested": 150.0}),
    # adjoint case: drop-in grid without tracers, 4 h at dt 120 s = 120 steps
    "adjoint": RunConfig("adjoint", 30, 4, 45, 0, 120.0, 120, "quadratic", extra={"dt_requested": 300.0}),
}
