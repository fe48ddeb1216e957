"""Several ranks on CPU (gloo, world size 2): the plumbing bench.py and the
sharded halo properties use on GPUs (one process per GPU over NCCL).

* partition_halos: contiguous runs of about equal cost, every halo once;
* gather_rows: each rank's rows reach rank 0 in halo order;
* max_over_ranks: timings are the slowest rank's;
* an end-to-end sharded reduction (the O(n) halo fields, computed per rank
  with the oracle's NumPy formulas) equals the single-process result exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ahop_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _catalogue():
    from ahop_b200 import synthetic
    return synthetic.halo_catalogue(60, seed=8, nmin=20, nmax=5000, box=100.0)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import halo_oracle
        off, pos, vel, mass, dens = _catalogue()
        b = replicas.partition_halos(off, world)
        loff, m0, m1 = replicas.local_members(off, b, rank)
        r = halo_oracle.props(loff, pos[m0:m1], vel[m0:m1], mass[m0:m1], dens[m0:m1], 100.0, 70.0, epot=False)
        rows = np.stack([r[f] for f in ["m", "px", "py", "pz", "r", "ek", "sigma"]], 1)
        full = replicas.gather_rows(rows, b, dist)
        slowest = replicas.max_over_ranks(float(rank + 1), dist)
        if rank == 0:
            q.put((full, slowest))
    finally:
        dist.destroy_process_group()


def test_partition_covers_every_halo_once_and_balances():
    off, *_ = _catalogue()
    for parts in (1, 2, 3, 8):
        b = replicas.partition_halos(off, parts)
        assert b[0] == 0 and b[-1] == len(off) - 1 and np.all(np.diff(b) >= 0)
    c = replicas.halo_cost(off)
    b = replicas.partition_halos(off, 2)
    share = [c[b[p]:b[p + 1]].sum() for p in range(2)]
    # no part exceeds half the total by more than the largest halo
    assert max(share) <= c.sum() / 2 + c.max()


def test_two_gloo_ranks_gather_and_max():
    import halo_oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, slowest = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    off, pos, vel, mass, dens = _catalogue()
    r = halo_oracle.props(off, pos, vel, mass, dens, 100.0, 70.0, epot=False)
    ref = np.stack([r[f] for f in ["m", "px", "py", "pz", "r", "ek", "sigma"]], 1)
    assert np.array_equal(full, ref)
    assert slowest == 2.0
