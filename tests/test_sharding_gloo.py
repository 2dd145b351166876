"""Multi-GPU host logic on CPU: the job scheduler that splits the mixed
workload across GPUs, and the rate aggregation (grid-point*steps summed,
elapsed time maxed over ranks), run as two gloo ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from paxpro_b200 import serving as sv
from paxpro_b200 import sharding as sh


def test_partition_covers_every_job_once_and_balances_work():
    jobs = sv.mixed_batch_jobs(seed=3)
    for world in (1, 2, 3, 8):
        parts = sh.partition_jobs(jobs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(jobs)))
        loads = [sum(sh.job_work(jobs[i]) for i in p) for p in parts]
        biggest = max(sh.job_work(j) for j in jobs)
        # greedy largest-first: no queue exceeds another by more than one job
        assert max(loads) - min(loads) <= biggest


def test_partition_is_deterministic_and_rejects_empty_world():
    jobs = sv.mixed_batch_jobs(seed=3)
    assert sh.partition_jobs(jobs, 4) == sh.partition_jobs(list(jobs), 4)
    with pytest.raises(ValueError):
        sh.partition_jobs(jobs, 0)


def test_device_bytes_by_precision():
    j2 = sv.Job("fft2d", 4096, 100, 0)
    j3 = sv.Job("fft3d", 1024, 100, 0)
    assert sh.job_device_bytes(j2, 0) == 4096 * 16 * 2
    assert sh.job_device_bytes(j3, 1) == 1024 * 1024 * 8 * 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = sv.mixed_batch_jobs(seed=3)
        mine = sh.partition_jobs(jobs, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        pts, secs = sh.reduce_rate(10.0 * (rank + 1), 1.0 + rank, dist)
        out[rank] = (gathered, pts, secs)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_split_and_aggregate_rates():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    jobs = sv.mixed_batch_jobs(seed=3)
    expect = sh.partition_jobs(jobs, world)
    for rank in range(world):
        gathered, pts, secs = out[rank]
        assert gathered == expect                      # every rank computed the same queues
        assert pts == 30.0 and secs == 2.0             # sum of work, max of time
