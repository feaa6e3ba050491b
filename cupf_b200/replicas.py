"""Replica plumbing of the multi-GPU run (one process per GPU, no data-path
collective): the simulation does not shard, so N GPUs run N independent replicas
and the job's throughput is the summed cell-updates over the slowest rank's
device time.  torch.distributed carries only the barrier and the max over ranks
(NCCL on GPUs, gloo on CPU for the tests)."""
from __future__ import annotations

import os


def dist_env():
    """(world size, rank, local rank) from the torchrun environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(pg, x, device="cpu"):
    """The largest of every rank's x (x itself without a process group)."""
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world_size, cells, steps, ms_max):
    """Whole-job cell-updates per second (millions): every replica advances
    `cells` cells by `steps` steps; the job takes the slowest rank's time."""
    return world_size * cells * steps / (ms_max / 1e3) / 1e6
