"""Shared set-up of parity cases: the oracle builds grid, metric and initial
state; the same arrays are handed to the CUDA library, so both sides see
identical inputs."""
import numpy as np

from cgd_b200 import grid as G
from cgd_b200 import physics as Ph


def grid_from_oracle(o, z, H, Rad):
    X, dX, J = o.metric()
    M, MM = o.mass()
    xw, w, DS, DW = o.gll()
    return G.Grid(o.nPanel, o.OrdPoly, o.nz, o.NF, o.NumG, o.NumNodes, o.NumEdges, Rad, H, np.asarray(z),
                  o.glob(), np.transpose(o.faces(), (2, 0, 1)), xw, w, DS, DW, X, dX, J, M, MM, o.dz())


def make_case(oracle_mod, nPanel, p, nz, NumTr, stretch="uniform", noise=0.01, H=30000.0, Rad=6.371e6):
    z = G.vertical_uniform(nz, H) if stretch == "uniform" else G.vertical_quadratic(nz, H)
    nu = Ph.hyperdiffusion(nPanel, p)
    o = oracle_mod.Oracle(nPanel, p, nz, NumTr, z, Rad=Rad, H=H, nu=nu, Up=1.0)
    tl = Ph.tracer_centres(NumTr, 20261204) if NumTr else None
    U = o.init_state(tl)
    Ph.theta_noise(U, noise, 20261203)
    return o, grid_from_oracle(o, z, H, Rad), U, nu


def rel_err_per_field(a, b):
    """max_i |a_i - b_i| / max_i |b_i| for every field (last axis)."""
    out = []
    for v in range(b.shape[-1]):
        den = np.abs(b[..., v]).max()
        num = np.abs(a[..., v] - b[..., v]).max()
        out.append(num / den if den > 0 else num)
    return np.array(out)
