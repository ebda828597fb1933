"""Multi-GPU plumbing for the explicit DG path: one process per GPU over torch.distributed.

The path shards without a data-path collective when the work is a set of independent solves (an
ensemble): instances are dealt to ranks so that each rank's element count is balanced, every rank
steps its own instances on its own GPU, and only the reporting needs a collective (the slowest
rank's time, the global conservation sums). A single mesh split across GPUs, with a halo exchange
of the ghost elements' coefficient blocks before every RK stage, is fve_dg_b200/partition.py.
"""
import numpy as np


def shard_instances(sizes, world):
    """Deal instances (with element counts `sizes`) to `world` ranks, largest first onto the
    least-loaded rank. Returns one sorted list of instance indices per rank; deterministic."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(x) for x in out]


def max_over_ranks(value, dist, device=None):
    """The largest of a per-rank float (the whole job's time is the slowest rank's)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def global_sums(local, dist, device=None):
    """Element-wise sum over ranks of per-rank conservation sums (mass, momentum, energy, ...)."""
    import torch
    t = torch.tensor(np.asarray(local, dtype=np.float64), device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()
