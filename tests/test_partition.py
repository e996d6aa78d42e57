"""Horizontal domain decomposition on the host (no GPU): the element
partition, each rank's halo plan, and the DSS exchange between two gloo
ranks.

Every rank packs the contributions of its boundary element nodes by its send
lists, exchanges them with TorchTransport (the transport the GPU path uses
over NCCL), unpacks them into its ghost slots and sums every local DOF's
contributors in the plan's order.  The oracle gives the element-node
contributions of the whole grid; the sums must equal its single-process DSS
(the phase-1 cache and the tendency) bit for bit, on both ranks."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from _cases import make_case  # noqa: E402


def _plans(glob, nranks):
    from cgd_b200.parallel import build_plans, partition_elements
    owner = partition_elements(glob.shape[1], nranks)
    return owner, build_plans(glob, owner)


@pytest.mark.parametrize("nranks", [2, 3, 8])
def test_plans_reproduce_the_global_owner_gather(oracle_mod, nranks):
    from cgd_b200.grid import inverse_map
    o, g, U, nu = make_case(oracle_mod, 4, 4, 3, 0)
    glob = g.glob
    DoF, NF = glob.shape
    owner, plans = _plans(glob, nranks)
    ptr, order = inverse_map(glob, g.NumG)
    count_owned = np.zeros(g.NumG, int)
    for P in plans:
        assert P.elems.size == np.sum(owner == P.rank)
        assert np.all(owner[P.elems] == P.rank)
        # boundary elements first: exactly those with a node another rank holds
        nb = P.nb_boundary
        if nranks > 1:
            assert 0 < nb <= P.NF
        # the local Glob addresses the same global DOFs
        assert np.array_equal(P.dofs[P.glob - 1], glob[:, P.elems] - 1)
        # every local DOF's contributor list is the global one, in order
        ghosts = {}
        for i, s in enumerate(P.neighbours):
            ghosts.update({slot: int(s) for slot in range(P.recv_ptr[i], P.recv_ptr[i + 1])})
        for lg, gg in enumerate(P.dofs):
            want = order[ptr[gg]:ptr[gg + 1]]
            got = P.contrib[P.contrib_ptr[lg]:P.contrib_ptr[lg + 1]]
            assert got.size == want.size
            for c, w in zip(got, want):
                e = int(w) // DoF
                if c >= 0:
                    assert P.elems[c // DoF] == e and c % DoF == w % DoF
                else:
                    assert owner[e] == ghosts[-1 - int(c)]
        count_owned[P.dofs[P.owned.astype(bool)]] += 1
        # ghost slots from neighbour s match what s sends here
        for i, s in enumerate(P.neighbours):
            Q = plans[int(s)]
            j = int(np.nonzero(Q.neighbours == P.rank)[0][0])
            assert P.recv_ptr[i + 1] - P.recv_ptr[i] == Q.send_ptr[j + 1] - Q.send_ptr[j]
    assert np.all(count_owned == 1)      # global sums count every DOF once


def _ordered_dss(P, Cloc, ghost):
    """Sum each local DOF's contributors in the plan's order (starting from
    0.0): Cloc (DoF, nf, nz, NF_local), ghost (n_ghost, nf, nz)."""
    DoF = P.DoF
    nf, nz = Cloc.shape[1], Cloc.shape[2]
    out = np.zeros((nz, P.NumG, nf), order="F")
    for lg in range(P.NumG):
        acc = np.zeros((nf, nz))
        for c in P.contrib[P.contrib_ptr[lg]:P.contrib_ptr[lg + 1]]:
            acc = acc + (Cloc[c % DoF, :, :, c // DoF] if c >= 0 else ghost[-1 - c])
        out[:, lg, :] = acc.T
    return out


def _exchange(P, transport, Cloc):
    """Pack this rank's send lists, exchange, return the ghost slots."""
    import torch
    DoF = P.DoF
    nf, nz = Cloc.shape[1], Cloc.shape[2]
    send = np.stack([Cloc[c % DoF, :, :, c // DoF] for c in P.send_list]) if P.send_list.size else \
        np.zeros((0, nf, nz))
    sbuf = torch.from_numpy(np.ascontiguousarray(send))
    rbuf = torch.zeros((P.n_ghost, nf, nz), dtype=torch.float64)
    sv = [sbuf[P.send_ptr[i]:P.send_ptr[i + 1]] for i in range(P.neighbours.size)]
    rv = [rbuf[P.recv_ptr[i]:P.recv_ptr[i + 1]] for i in range(P.neighbours.size)]
    transport.exchange(sv, rv)
    return rbuf.numpy()


def _gloo_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "cgdycore.jl_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import oracle
        from cgd_b200.parallel import TorchTransport
        o, g, U, nu = make_case(oracle, 4, 4, 6, 1, "quadratic")
        _, plans = _plans(g.glob, world)
        P = plans[rank]
        T = TorchTransport(P)
        # phase 1: contributions of the local elements only, exchanged
        C1 = o.contributions(U)
        t1 = _ordered_dss(P, C1[..., P.elems], _exchange(P, T, C1[..., P.elems]))
        T1 = o.hypervisc1(U)
        ok1 = np.array_equal(t1, T1[:, P.dofs, :])
        # phase 2 at the DSS'd cache
        C2 = o.contributions(U, T1)
        f = _ordered_dss(P, C2[..., P.elems], _exchange(P, T, C2[..., P.elems]))
        ok2 = np.array_equal(f, o.rhs(U)[:, P.dofs, :])
        # the global mass integral from the ranks' partial sums (each DOF on its owner)
        from cgd_b200.parallel import global_mass_integral
        MM = np.asarray(P.local_grid(g).MMass)
        part = float((U[:, P.dofs, 0] * MM).sum())
        tot = global_mass_integral(part)
        ok3 = abs(tot - o.mass_integral(U)) <= 1e-13 * abs(o.mass_integral(U))
        with open(os.path.join(out, f"r{rank}.txt"), "w") as fh:
            fh.write(f"{int(ok1)} {int(ok2)} {P.n_ghost} {P.send_list.size} {int(ok3)}")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_dss_matches_single_process(tmp_path, oracle_mod):
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_gloo_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        ok1, ok2, ng, ns, ok3 = open(tmp_path / f"r{r}.txt").read().split()
        assert ok1 == "1", f"rank {r}: phase-1 DSS differs from the single-process one"
        assert ok2 == "1", f"rank {r}: tendency differs from the single-process one"
        assert ok3 == "1", f"rank {r}: the all-reduced mass integral differs from the single-process one"
        assert int(ng) > 0 and int(ns) > 0
