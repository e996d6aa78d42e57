"""Horizontal domain decomposition of the spectral-element grid: element
partition, the per-rank halo plan of the direct-stiffness summation (DSS) and
the transport of its exchanges.

The reference partitions the faces of the cubed sphere over MPI ranks
(``Grids.Decompose`` / ``DecomposeEqualArea``, src/Grids/InitGrid.jl:34-43),
builds each rank's sub-grid with its boundary faces first
(``ConstructSubGridGhost``, src/Grids/SubGridGhost.jl:48-73) and, after each
of the two DSS points of a tendency, adds the boundary values received from
its neighbours (``ExchangeData3DSendGPU`` / ``ExchangeData3DRecvGPU!``,
src/Parallels/Exchange.jl:938-1071; src/GPU/FcnGPU.jl:777-913).

Here a rank exchanges element-node *contributions*, not partial sums: every
rank that holds a DOF receives the contributions of the element nodes that
other ranks own at that DOF, and sums all of them in ascending global
(element, node) order - the order of the single-process owner gather.  So
the DSS'd values, and the column solves that follow, are bit for bit the
single-process ones on every rank, and shared columns stay consistent
without exchanging the state.

  partition_elements(NF, nranks)   contiguous ranges of the element order
  HaloPlan                         one rank's local grid and exchange lists
  build_plans(grid, owner)         the plans of every rank
  TorchTransport                   the exchange over torch.distributed
                                   (NCCL between GPUs, gloo on the host)
"""
from dataclasses import dataclass

import numpy as np

from .grid import Grid, inverse_map


def partition_elements(NF, nranks):
    """Owner rank of every element: nranks contiguous ranges of the element
    order (the cubed sphere numbers its elements panel by panel, row by row,
    so a range is one or a few compact bands of a panel), of equal size to
    within one element - an equal-area partition, as every element of the
    equiangular cubed sphere has nearly the same area."""
    if nranks < 1 or nranks > NF:
        raise ValueError("need 1 <= nranks <= NF")
    bounds = (np.arange(nranks + 1, dtype=np.int64) * NF) // nranks
    owner = np.zeros(NF, np.int32)
    for r in range(nranks):
        owner[bounds[r]:bounds[r + 1]] = r
    return owner


@dataclass
class HaloPlan:
    """What rank ``rank`` holds and exchanges.

    elems        global element ids of the local elements, boundary elements
                 first (those with a node that another rank also holds),
                 each group ascending (SubGridGhost.jl:71 orders [B; I])
    nb_boundary  number of boundary elements at the front of ``elems``
    dofs         global DOF ids (0-based) of the local DOFs, ascending
    glob         (DoF, NF_local) int64, 1-based local DOF ids
    contrib_ptr  (NumG_local + 1,) CSR offsets
    contrib      contributors of each local DOF in ascending global (element,
                 node) order: c >= 0 is the local element node
                 (local element * DoF + node), c < 0 the ghost slot -1 - c
    neighbours   ranks sharing a DOF with this one, ascending
    send_ptr     (len(neighbours) + 1,) offsets into send_list
    send_list    local element nodes whose contribution goes to each
                 neighbour, in that neighbour's ghost-slot order
    recv_ptr     (len(neighbours) + 1,): ghost slots recv_ptr[i] ..
                 recv_ptr[i+1]-1 are filled from neighbours[i]
    owned        (NumG_local,) uint8: 1 where this rank is the lowest rank
                 holding the DOF (it counts the DOF in global sums, the
                 reference's MasterSlave, SubGridGhost.jl:92-99)
    """
    rank: int
    nranks: int
    DoF: int
    elems: np.ndarray
    nb_boundary: int
    dofs: np.ndarray
    glob: np.ndarray
    contrib_ptr: np.ndarray
    contrib: np.ndarray
    neighbours: np.ndarray
    send_ptr: np.ndarray
    send_list: np.ndarray
    recv_ptr: np.ndarray
    owned: np.ndarray

    @property
    def NF(self):
        return int(self.elems.size)

    @property
    def NumG(self):
        return int(self.dofs.size)

    @property
    def n_ghost(self):
        return int(self.recv_ptr[-1])

    # ---- restriction of the global arrays to this rank
    def local_grid(self, grid):
        """The rank's grid: its elements' metric and its DOFs' mass and dz,
        taken from the global arrays (so dz and M are the single-process
        values at shared columns), and the local Glob."""
        e, d = self.elems, self.dofs
        mm = np.asfortranarray(grid.MMass[:, d] * self.owned[None, :])   # global sums count each DOF once
        return Grid(grid.nPanel, grid.OrdPoly, grid.nz, self.NF, self.NumG, 0, 0, grid.Rad, grid.H, grid.z,
                    np.asfortranarray(self.glob), grid.faces[e], grid.xw, grid.w, grid.DS, grid.DW,
                    np.asfortranarray(grid.X[..., e]), np.asfortranarray(grid.dXdxI[..., e]),
                    np.asfortranarray(grid.J[..., e]), np.asfortranarray(grid.M[:, d, :]), mm,
                    np.asfortranarray(grid.dz[:, d]))

    def restrict(self, U):
        """The rank's part of a global state (nz, NumG, NV)."""
        return np.asfortranarray(U[:, self.dofs, :])


def build_plans(grid_or_glob, owner):
    """The halo plan of every rank for the element owners ``owner`` (NF,).
    Every rank can build all plans (they are cheap), so the send lists of one
    rank and the ghost slots of its neighbours agree by construction."""
    glob = grid_or_glob.glob if hasattr(grid_or_glob, "glob") else grid_or_glob
    glob = np.asarray(glob)
    DoF, NF = glob.shape
    numg = int(glob.max())
    owner = np.asarray(owner, np.int64)
    nranks = int(owner.max()) + 1
    ptr, order = inverse_map(glob, numg)            # contributors IF*DoF+ID of each DOF, ascending
    cnt = np.diff(ptr)
    c_elem = order // DoF
    c_rank = owner[c_elem]
    dof_of_c = np.repeat(np.arange(numg), cnt)
    # ranks holding each DOF (a DOF is held by every rank with a contributor)
    held = [set() for _ in range(nranks)]            # DOFs per rank
    dof_ranks = {}
    for g, r in zip(dof_of_c, c_rank):
        dof_ranks.setdefault(int(g), set()).add(int(r))
    for g, rs in dof_ranks.items():
        for r in rs:
            held[r].add(g)
    plans = []
    # ghost-slot order of rank r for contributions from rank s: the global
    # (element, node) order of the contributors that s owns at DOFs r holds
    ghost = {}                                       # (r, s) -> array of contributor ids (IF*DoF+ID)
    for r in range(nranks):
        mine = np.zeros(numg, bool)
        mine[list(held[r])] = True
        sel = mine[dof_of_c] & (c_rank != r)
        for s in np.unique(c_rank[sel]):
            cs = order[sel & (c_rank == s)]
            ghost[(r, int(s))] = np.sort(cs)
    for r in range(nranks):
        dofs = np.array(sorted(held[r]), np.int64)
        loc = np.full(numg, -1, np.int64)
        loc[dofs] = np.arange(dofs.size)
        el = np.nonzero(owner == r)[0]
        # boundary elements: a node held by another rank too
        shared = np.array([len(dof_ranks[g]) > 1 for g in range(numg)], bool)
        gl = glob[:, el] - 1
        is_b = shared[gl].any(axis=0)
        elems = np.concatenate([el[is_b], el[~is_b]])
        eloc = np.full(NF, -1, np.int64)
        eloc[elems] = np.arange(elems.size)
        lglob = loc[glob[:, elems] - 1] + 1
        nbs = np.array(sorted(s for (rr, s) in ghost if rr == r), np.int64)
        # ghost slots: neighbour by neighbour
        slot_of = {}
        recv_ptr = [0]
        for s in nbs:
            for c in ghost[(r, int(s))]:
                slot_of[int(c)] = len(slot_of)
            recv_ptr.append(len(slot_of))
        # contributor lists of the local DOFs
        cptr = [0]
        clist = []
        for g in dofs:
            for c in order[ptr[g]:ptr[g + 1]]:
                e = int(c) // DoF
                if owner[e] == r:
                    clist.append(int(eloc[e]) * DoF + int(c) % DoF)
                else:
                    clist.append(-1 - slot_of[int(c)])
            cptr.append(len(clist))
        # send lists: what each neighbour s expects from r, in s's slot order
        send_ptr = [0]
        slist = []
        for s in nbs:
            for c in ghost[(int(s), r)]:
                slist.append(int(eloc[int(c) // DoF]) * DoF + int(c) % DoF)
            send_ptr.append(len(slist))
        owned = np.array([min(dof_ranks[int(g)]) == r for g in dofs], np.uint8)
        plans.append(HaloPlan(r, nranks, DoF, elems.astype(np.int64), int(is_b.sum()), dofs,
                              np.asfortranarray(lglob.astype(np.int64)), np.array(cptr, np.int32),
                              np.array(clist, np.int32), nbs.astype(np.int32), np.array(send_ptr, np.int32),
                              np.array(slist, np.int32), np.array(recv_ptr, np.int32), owned))
    return plans


class TorchTransport:
    """The DSS exchange over a torch.distributed process group: for every
    neighbour one send of this rank's packed contributions and one receive of
    the neighbour's, issued together (batch_isend_irecv) and waited for.
    Works on CUDA tensors (NCCL: each transfer is one peer send/receive over
    NVLink) and on host tensors (gloo)."""

    def __init__(self, plan, group=None):
        self.plan = plan
        self.group = group

    def exchange(self, send_views, recv_views):
        """send_views[i] goes to plan.neighbours[i], recv_views[i] is filled
        from it."""
        import torch.distributed as dist
        ops = []
        for i, s in enumerate(self.plan.neighbours):
            ops.append(dist.P2POp(dist.isend, send_views[i], int(s), group=self.group))
            ops.append(dist.P2POp(dist.irecv, recv_views[i], int(s), group=self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


def global_mass_integral(local, group=None, device=None):
    """Parallels.GlobalIntegral (src/Parallels/Exchange.jl:1163-1166) over a
    decomposed grid: the sum over the ranks of each rank's mass integral
    (`local`, e.g. Dycore.mass_integral of the rank's part, whose MMass
    counts a DOF on its owner only; HaloPlan.local_grid), by one FP64
    all-reduce.  device: where the reduced value lives (a CUDA device for
    NCCL, None for host tensors with gloo).  The order of the ranks' partial
    sums is the collective's, so the result agrees with a single-process sum
    to rounding."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
