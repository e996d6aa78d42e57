"""Gradients of scalar functionals of a Rosenbrock-W run, through the
hand-written adjoints of the library (cgd_ros_step_adjoint chained over
checkpoints by Dycore.steps_adjoint).

BoxPressureFunctional is the sensitivity target of the adjoint workload: the
mean, over the columns whose lowest-layer midpoint lies in a latitude /
longitude box, of the squared anomaly of the lowest-layer pressure p1 (the
path's surface-pressure proxy; the reference has no surface-pressure
diagnostic on this path) after n steps against the initial state:

    J(U0) = mean_box (p1(U_n) - p1(U0))^2,   U_n = step^n(U0).

Pressure is p = p0 (Rd rho*theta / p0)^(1/(1-kappa)) (PressureKernel!,
src/GPU/DiagnosticKernel.jl:96-115), so dp/d(rho*theta) = p / ((1-kappa) rho*theta).
"""
import numpy as np


def column_lonlat(grid):
    """Longitude in [0, 2 pi) and latitude (radians) of the lowest-layer
    midpoint of every column; a column's node takes the coordinates of the
    highest-numbered element that holds it, as the initial state does."""
    from .grid import node_positions
    P = node_positions(grid)                                       # (numg, 2, 3, nz)
    mid = 0.5 * (P[:, 0, :, 0] + P[:, 1, :, 0])                    # (numg, 3)
    lon = np.mod(np.arctan2(mid[:, 1], mid[:, 0]), 2 * np.pi)
    lat = np.arcsin(mid[:, 2] / np.linalg.norm(mid, axis=1))
    return lon, lat


def box_columns(grid, lat_deg=(45.0, 55.0), lon_deg=(55.0, 65.0)):
    lon, lat = column_lonlat(grid)
    lat, lon = np.degrees(lat), np.degrees(lon)
    return np.nonzero((lat >= lat_deg[0]) & (lat <= lat_deg[1]) & (lon >= lon_deg[0]) & (lon <= lon_deg[1]))[0]


class BoxPressureFunctional:
    """J(U0) = mean over the box columns of (p1(U_n) - p1(U0))^2 for a
    Dycore d, n steps of size dt.  States are device (torch) or host (numpy)
    arrays as Dycore accepts them."""

    def __init__(self, d, dt, nsteps, box=None, every=None):
        self.d, self.dt, self.n, self.every = d, float(dt), int(nsteps), every
        self.box = box_columns(d.grid) if box is None else np.asarray(box)
        self.kappa = d.phys.kappa

    def _p1(self, V):
        return np.asarray(self.d.fcn_prepare(V))[0][self.box].copy()

    def _rth1(self, V):
        if isinstance(V, np.ndarray):
            return V[0, self.box, 4].copy()
        import torch
        return V[4, torch.as_tensor(self.box, device=V.device), 0].cpu().numpy()

    def _run(self, U0, work=None):
        V = U0.copy(order="F") if isinstance(U0, np.ndarray) else (U0.clone() if work is None else work.copy_(U0))
        self.d.time_stepper(V, self.dt, self.n)
        return V

    def anomaly(self, U0, work=None):
        """p1(U_n) - p1(U0) on the box columns (and U_n)."""
        Un = self._run(U0, work)
        return self._p1(Un) - self._p1(U0), Un

    def value(self, U0, work=None):
        A, _ = self.anomaly(U0, work)
        return float(np.mean(A * A))

    def diff(self, Up, Um, work=None):
        """J(Up) - J(Um), formed from the anomalies entry by entry."""
        Ap, _ = self.anomaly(Up, work)
        Am, _ = self.anomaly(Um, work)
        return float(np.mean((Ap - Am) * (Ap + Am)))

    def _seed(self, V, coef):
        """An array like V, zero except rho*theta of the lowest layer of the
        box columns: coef * dp/d(rho*theta) there."""
        p = self._p1(V)
        val = coef * p / ((1.0 - self.kappa) * self._rth1(V))
        if isinstance(V, np.ndarray):
            S = np.zeros_like(V, order="F")
            S[0, self.box, 4] = val
            return S
        import torch
        S = torch.zeros_like(V)
        S[4, torch.as_tensor(self.box, device=V.device), 0] = torch.from_numpy(val).to(V.device)
        return S

    def value_and_grad(self, U0):
        """J(U0) and dJ/dU0 (an array like U0), from one forward run (which
        keeps the checkpoints) and the reverse sweep."""
        p10 = self._p1(U0)
        out = {}

        def seed(Un):
            out["A"] = A = self._p1(Un) - p10
            return self._seed(Un, 2.0 / self.box.size * A)

        G = self.d.steps_adjoint(U0, seed, self.dt, self.n, every=self.every)
        A = out["A"]
        G -= self._seed(U0, 2.0 / self.box.size * A)   # J depends on U0 through p1(U0) too
        return float(np.mean(A * A)), G
