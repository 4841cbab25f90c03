"""Energy sharding across ranks (world size 2, gloo on CPU).

Each rank integrates the contiguous range of energy points that the library's
negf_shard_range assigns to it (here with the CPU oracle standing in for the
device pass, since this runs without a GPU), the partial site charges are
summed with one all-reduce, and Rho0 is subtracted once.  The result must equal
the single-rank charge.
"""
import os
import socket

import numpy as np
import pytest

CASE = dict(type_id=(17, 0), num_unitcells=8, num_modes=2, contact_mu=(0.0, -0.3), contact_T=(300.0, 300.0),
            eq_integration_pts=(12, 12, 16), noneq_integration_pts=(50,))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime

    import torch
    import torch.distributed as dist
    from electrostatic_b200.negf import shard_range
    from oracle import oracle as O

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    t = O.OracleTube(**CASE)
    y = np.linspace(0, 1, t.N)
    U = 0.2 * np.sin(6 * y) + 0.1 * y
    t.set_potential(U, (U[0], U[-1]))
    n_eq = len(t.paths(1)[0])
    n_ne = len(t.paths(3)[0])
    lo, hi = shard_range(n_eq + n_ne, rank, world)
    part = np.zeros(t.N)
    if lo < n_eq:
        part += t.partial(1, lo, min(hi, n_eq))
    if hi > n_eq:
        part += t.partial(3, max(lo, n_eq) - n_eq, hi - n_eq)
    Q = torch.tensor(part)
    dist.all_reduce(Q)  # the one exchange of the path: N doubles per pass
    if rank == 0:
        _, _, _, rho0 = t.charge(components=True)
        q.put((Q.numpy() - rho0, t.charge()))
    dist.barrier()
    dist.destroy_process_group()


def test_energy_shards_allreduce_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, full = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    np.testing.assert_allclose(got, full, rtol=1e-12, atol=1e-14 * np.abs(full).max())
