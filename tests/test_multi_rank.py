"""The multi-GPU path of bench.py (independent replicas, max-over-ranks timing) as two gloo ranks
on CPU: every rank takes the same collective steps, the reported time is the slowest rank's, the
whole-job rate counts every rank's units, replicas trace different ray sets, and the reference
arm runs on rank 0 only."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from liar_b200 import scenes


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench.dist_setup()
        assert (w, r, local) == (world, rank, rank)
        ms = 10.0 + 5.0 * rank                      # rank 1 is the slower one
        slowest = bench.max_over_ranks(ms, w, dist, "cpu")
        v, f = scenes.displaced_icosphere(2, seed=0)
        rays = scenes.random_rays(v, 64, seed=bench.replica_seed(r))
        out[rank] = (slowest, bench.whole_job_rate(w, 1000, slowest), float(rays[:, :3].sum()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_replicas():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0               # both report the slowest rank's time
    assert res[0][1] == pytest.approx(2 * 1000 / 15e-3)  # all ranks' units over that time
    assert res[0][2] != res[1][2]                       # replicas trace different rays


def test_single_rank_is_identity():
    assert bench.max_over_ranks(3.5, 1, None, "cpu") == 3.5
    assert bench.whole_job_rate(1, 500, 2.0) == pytest.approx(250000.0)


def test_reference_arm_only_on_rank_zero(capsys):
    class A:
        warmup, steps = 0, 1
    bench.run_reference(A(), 2, 1)
    assert capsys.readouterr().out == ""
