"""The N>1 path on CPU: two gloo ranks, each with its own workload (weak
scaling, no data-path collective), time reduced as the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from n2p2_b200 import ranks, water
    r, w, _ = ranks.rank_env()
    batch = water.water_batch(4, seed=ranks.rank_seed(1, r))
    natoms = sum(s.numAtoms for s in batch)
    t = ranks.max_over_ranks(10.0 + r)          # pretend rank r took 10 + r ms
    total = ranks.sum_over_ranks(natoms)
    out[r] = (natoms, t, total, float(batch[0].positions[0, 0]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_weak_scaling_and_max_time():
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    (n0, t0, tot0, x0), (n1, t1, tot1, x1) = res[0], res[1]
    assert t0 == t1 == 11.0                     # max over ranks
    assert tot0 == tot1 == n0 + n1              # job-wide atom count
    assert x0 != x1                             # each rank has its own structures
