"""The N > 1 path of bench.py on CPU: world_size-2 gloo process groups (no GPU).

The simulation does not shard ("replicas only"): each rank runs its own copy and
the only collectives are the barrier and the max over ranks of the timed
region.  These tests run that plumbing (cupf_b200/replicas.py, the functions
bench.py calls) across two processes, and check that the reference arm does its
work on rank 0 only.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from cupf_b200.replicas import dist_env, max_over_ranks, replica_throughput
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    assert dist_env() == (ws, rank, rank)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    dist.barrier()
    # rank r "timed" 10 + 5 r ms for 100 steps of a 1000-cell replica
    ms = max_over_ranks(dist, 10.0 + 5.0 * rank, "cpu")
    value = replica_throughput(ws, 1000, 100, ms)
    with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
        f.write("%r %r\n" % (ms, value))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_throughput_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    ws = 2
    mp.start_processes(_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, join=True,
                       start_method="spawn")
    for r in range(ws):
        ms, value = (float(v) for v in open(tmp_path / ("rank%d.txt" % r)).read().split())
        assert ms == 15.0  # every rank sees the slowest rank's time
        # two replicas x 1000 cells x 100 steps in 15 ms
        assert value == pytest.approx(2 * 1000 * 100 / 15e-3 / 1e6)


def test_single_process_without_group():
    sys.path.insert(0, ROOT)
    from cupf_b200.replicas import max_over_ranks, replica_throughput
    assert max_over_ranks(None, 3.5) == 3.5
    assert replica_throughput(1, 10, 2, 1.0) == pytest.approx(0.02)


def test_reference_arm_runs_on_rank0_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup, gpus = 1, 0, 2
    assert bench.run_reference(Args(), 2, 1) == 0
    assert capsys.readouterr().out == ""
