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


def ordered_dss(C, glob, NumG):
    """Owner gather of element-node contributions C (DoF, nf, nz, NF): every
    DOF sums its contributors in ascending (element, node) order, starting
    from 0.0; result (nz, NumG, nf)."""
    DoF, nf, nz, NF = C.shape
    out = np.zeros((nz, NumG, nf), order="F")
    acc = np.zeros((NumG, nf, nz))
    for IF in range(NF):
        for ID in range(DoF):
            g = int(glob[ID, IF]) - 1
            acc[g] = acc[g] + C[ID, :, :, IF]
    out[:] = np.transpose(acc, (2, 0, 1))
    return out


def merge_dofs(o, g, U, A, B):
    """A grid whose DOF B (0-based) is merged into DOF A, so that A gathers
    the contributors of both (five or more where A has four).  The oracle is
    given B's copy of A's mass and the state B's copy of A's column, so its
    element-node contributions are those of the merged grid.  Returns the
    merged grid, its state and the state with B's column set to A's (for the
    oracle)."""
    import dataclasses
    NumG = g.NumG
    keep = np.array([k for k in range(NumG) if k != B])
    new = np.empty(NumG, np.int64)
    new[keep] = np.arange(NumG - 1)
    new[B] = new[A]
    M, MM = o.mass()
    M2 = np.array(M, order="F")
    M2[:, B, :] = M[:, A, :]
    o.set_metric(M=M2)
    Uo = np.array(U, order="F")
    Uo[:, B, :] = U[:, A, :]
    glob2 = np.asfortranarray(new[np.asarray(g.glob) - 1] + 1, dtype=np.int64)
    g2 = dataclasses.replace(g, NumG=NumG - 1, glob=glob2, M=np.asfortranarray(M2[:, keep, :]),
                             MMass=np.asfortranarray(np.asarray(MM)[:, keep]),
                             dz=np.asfortranarray(np.asarray(g.dz)[:, keep]))
    return g2, np.asfortranarray(Uo[:, keep, :]), Uo
