"""CPU: multi-rank plumbing over gloo with world_size 2 (the N>1 path of the ensemble sharding)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fve_dg_b200 import box_mesh
from fve_dg_b200.distributed import global_sums, max_over_ranks, shard_instances
from oracle.pyoracle import Oracle


def test_shard_instances_balanced_and_complete():
    rng = np.random.default_rng(0)
    sizes = [6 * int(n) ** 3 for n in rng.integers(8, 33, 64)]
    for world in (1, 2, 4, 8):
        parts = shard_instances(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
        assert parts == shard_instances(sizes, world)  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [2, 3, 2, 3]
        mine = shard_instances([6 * n ** 3 for n in sizes], world)[rank]
        # each rank "steps" its own instances: here, the oracle's conservation sums of their states
        sums = np.zeros(6)
        for i in mine:
            m = box_mesh(sizes[i], jitter=0.05, seed=i)
            o = Oracle.from_mesh(m)
            U = np.zeros((m.ncell, 20))
            U[:, 0] = 1.0 + 0.1 * i
            U[:, 4] = 2.5
            sums += o.conservation(U, 1, 0)
        tot = global_sums(sums, dist)
        slow = max_over_ranks(float(rank + 1), dist)
        q.put((rank, mine, tot.tolist(), slow))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_ensemble_sums_over_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=90) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    res.sort()
    assert sorted(res[0][1] + res[1][1]) == [0, 1, 2, 3]
    assert res[0][2] == res[1][2]  # every rank sees the same global sums
    assert res[0][3] == res[1][3] == 2.0  # the slowest rank's value
    # the global mass equals the sum over all instances of (mean density) x (box volume 1)
    assert np.isclose(res[0][2][0], sum(1.0 + 0.1 * i for i in range(4)), rtol=1e-12)
