"""Energy shards through the library on the GPU, summed across processes.

Two processes (world size 2, gloo on the host) each create the same tube on
cuda:0, restrict it to their shard of the energy points with
negf_tube_set_energy_shard (Rho0 subtracted on rank 0 only), compute their
partial charge with the sm_100a kernels and sum the partials with one
all-reduce of N doubles -- the one exchange of the multi-GPU data plane.  The
sum must equal the FP64 oracle's full charge.  The ranks' kernels never wait
on each other (each launch is independent), so sharing one GPU is safe.
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASE = dict(type_id=(17, 0), num_unitcells=120, num_modes=4, contact_mu=(0.0, -0.4), contact_T=(300.0, 300.0),
            eq_integration_pts=(32, 32, 64), noneq_integration_pts=(150, 300, 150),
            noneq_percent_intercuts=(30.0, 70.0))


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
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.workloads import site_potential

    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = CNT(**CASE)
        U = site_potential(t.site_positions(), 4242)
        t.set_potential(U, (U[0], U[-1]))
        t.set_energy_shard(rank, world)
        part = torch.from_numpy(t.Solve_NEGF())  # this rank's partial charge (host)
        dist.all_reduce(part)  # N doubles: the one exchange per pass
        if rank == 0:
            q.put((part.numpy(), U))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_energy_shards_on_gpu_sum_to_oracle(oracle):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, U = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    o = oracle.OracleTube(**CASE)
    o.set_potential(U, (U[0], U[-1]))
    full = o.charge(nthreads=8)
    err = np.max(np.abs(got - full)) / np.max(np.abs(full))
    assert err <= 1e-8, err
