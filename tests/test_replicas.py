"""bench.py's multi-rank mode on CPU: two processes over the gloo backend.

The path runs replicas only (one independent solve per GPU, no data-path
collective); what crosses ranks is the timing: the whole job's time of a timed
region is the largest rank's (an all-reduce MAX that every rank takes, in the
same order), and the reference arm runs on rank 0 alone.
"""
import argparse
import datetime
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        # the solve timing, then the end-to-end timing, as bench.main takes them
        t = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        e = bench.max_over_ranks(20.0 - rank, dist, "cpu")
        out[rank] = (t, e, bench.replica_value(1000, 4, world, t))
    finally:
        dist.destroy_process_group()


def test_job_time_is_the_largest_rank_time():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]
    t, e, v = res[0]
    assert t == 15.0 and e == 20.0
    # every replica solved 1000 unknowns in each of 4 steps within 15 ms
    assert v == 1000 * 4 * world / 15e-3


def test_single_rank_keeps_its_own_time():
    import bench
    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.replica_value(274625, 5, 1, 7.7) == 274625 * 5 / 7.7e-3


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import bench
    args = argparse.Namespace(gpus=2, steps=1, warmup=0)
    bench.run_reference_arm(args, 2, 1)
    assert capsys.readouterr().out == ""
