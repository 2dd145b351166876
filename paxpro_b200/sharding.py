"""Independent propagation jobs across GPUs: one process per GPU, no data-path
collective.

The mixed and served workloads are sets of independent jobs (one field each),
so they shard by job: a host-side scheduler gives every GPU its own queue,
filled greedily with the largest remaining job going to the least-loaded GPU
(longest-processing-time first), load measured as grid-point*steps.  Each
rank then runs its queue alone (batched or served) and results stay on that
rank's host.  The only collectives are the host-side aggregation of the
measured rates: grid-point*steps summed over ranks and the elapsed time taken
as the maximum over ranks, on whatever process group the caller set up
(NCCL between GPUs, gloo on CPU in tests).

A single field is not sharded (a split 2-D FFT would need an all-to-all
transpose every step): one field, one GPU.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def job_work(job) -> float:
    """Grid-point*steps of a job (the load the scheduler balances)."""
    return float(job.pts_steps)


def job_device_bytes(job, precision: int) -> int:
    """Device bytes a job's field and its ping-pong copy need (complex128 in
    FP64 mode, complex64 in FP32); tables are small beside them."""
    pts = job.n * job.n if job.kind == "fft3d" else job.n
    return pts * (16 if precision == 0 else 8) * 2


def partition_jobs(jobs: Sequence, world: int) -> List[List[int]]:
    """Indices of `jobs` per rank: largest job first onto the least-loaded
    rank (ties: lower rank).  Deterministic, so every rank computes the same
    split without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(jobs)), key=lambda i: (-job_work(jobs[i]), i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += job_work(jobs[i])
    for q in out:
        q.sort()
    return out


def reduce_rate(pts_steps: float, seconds: float, dist=None, device=None) -> Tuple[float, float]:
    """(sum of grid-point*steps, max of elapsed seconds) over the ranks of the
    default process group; the local values when `dist` is None."""
    if dist is None:
        return float(pts_steps), float(seconds)
    import torch
    t = torch.tensor([float(pts_steps)], dtype=torch.float64, device=device)
    m = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(t.item()), float(m.item())
