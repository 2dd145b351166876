"""Batched and served propagation on one GPU.

Job streams with the parameter distributions of the mixed-workload
configurations:

  * 2-D jobs (one transverse dim): FFTSolver2D or CrankNicholson, Nx a power
    of two drawn log-uniformly, steps uniform in [200, 5000], a planar
    waveguide (core half-width U[10, 60] nm, cladding delta U[2e-6, 3e-5],
    beta = delta/80, 25-point beta ramp at the edges), Gaussian waist
    U[5, 30] nm, wavelength 0.1 nm, x in [-250, 250] nm;
  * 3-D jobs: FFTSolver3D, Nx = Ny in {256, 512, 1024, 2048} on
    [-1000, 1000]^2 nm, steps of 2 um, a unit plane wave and 8 seeded
    spheres (radius U[20, 150], centre uniform in the volume, delta
    U[1e-6, 5e-5], beta = delta/50).

Every size is drawn as stated: FFTSolver2D lines of 16384 complex128 points
run on a cluster of two CTAs, CrankNicholson systems of 8192 and 16384 rows
on clusters of two and four CTAs (the step-invariant path of the
waveguides' z-invariant media).

`run_batched` admits every job into one Batch (one launch per group of equal
2-D kind/size, 3-D jobs on their own streams); `run_plain` runs the same jobs
one at a time through single solver handles; `serve` is the request loop:
Poisson arrivals, admission by device-memory budget, fields resident on the
device between rounds, new jobs slotted in as others finish, exit intensity
returned per job, p50/p99 latency reported.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

import paxpro_b200 as pxp
from paxpro_b200 import workloads as wl

MAX_FFT2D_N = 16384
MAX_CN_N = 16384


@dataclass
class Job:
    kind: str                  # "fft2d" | "cn" | "fft3d"
    n: int
    nsteps: int
    seed: int
    core_half_width: float = 25.0
    delta_clad: float = 7.5e-6
    waist: float = 15.0
    spheres: List[tuple] = field(default_factory=list)
    arrival: float = 0.0       # seconds, serving only

    @property
    def pts_steps(self) -> float:
        return float(self.n if self.kind != "fft3d" else self.n * self.n) * self.nsteps


def draw_2d(rng: np.random.Generator, kind: str, seed: int) -> Job:
    n = min(2 ** int(rng.integers(8, 15)), MAX_FFT2D_N if kind == "fft2d" else MAX_CN_N)
    steps = int(rng.integers(200, 5001))
    core = float(rng.uniform(10.0, 60.0))
    delta = float(rng.uniform(2e-6, 3e-5))
    waist = float(rng.uniform(5.0, 30.0))
    return Job(kind, n, steps, seed, core, delta, waist)


def draw_3d(rng: np.random.Generator, seed: int, sizes=(256, 512, 1024, 2048)) -> Job:
    n = int(rng.choice(sizes))
    steps = int(rng.integers(200, 5001))
    sph = wl.random_spheres(rng, 8, -1000.0, 1000.0, steps * 2000.0)
    return Job("fft3d", n, steps, seed, spheres=sph)


def mixed_batch_jobs(seed: int = 3, n2d: int = 512, n3d: int = 32) -> List[Job]:
    """512 2-D problems (80 % FFT, 20 % CN) plus 32 3-D FFT problems."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n2d):
        kind = "fft2d" if rng.random() < 0.8 else "cn"
        jobs.append(draw_2d(rng, kind, i))
    for i in range(n3d):
        jobs.append(draw_3d(rng, n2d + i))
    return jobs


def served_jobs(rate: float, duration: float, seed: int = 4) -> List[Job]:
    """Poisson arrivals at `rate` jobs/s for `duration` s: 80 % 2-D FFT,
    15 % CN, 5 % 3-D FFT (N <= 2048)."""
    rng = np.random.default_rng(seed)
    t, jobs, i = 0.0, [], 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        u = rng.random()
        job = draw_2d(rng, "fft2d", i) if u < 0.80 else (
            draw_2d(rng, "cn", i) if u < 0.95 else draw_3d(rng, i))
        job.arrival = t
        jobs.append(job)
        i += 1
    return jobs


def make_solver(job: Job, precision: int, device: int = 0) -> pxp.Solver:
    """A solver handle with material and initial field set."""
    if job.kind == "fft3d":
        xmin, xmax = -1000.0, 1000.0
        dx = wl.step_for_nodes(xmin, xmax, job.n)
        dz = 2000.0
        spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_3D, x=pxp.Disc(xmin, xmax, dx),
                               y=pxp.Disc(xmin, xmax, dx),
                               z=pxp.Disc(0.0, job.nsteps * dz, dz), wavenumber=wl.K,
                               precision=precision, device=device)
        s = pxp.Solver(spec)
        s.set_material_spheres([pxp.Sphere(*sp) for sp in job.spheres])
        s.set_initial_conditions(np.ones((job.n, job.n), dtype=np.complex128, order="F"))
        return s
    xmin, xmax = -250.0, 250.0
    dx = wl.step_for_nodes(xmin, xmax, job.n)
    dz = 1000.0 if job.kind == "fft2d" else 500.0
    guide = wl.Waveguide(core_half_width=job.core_half_width, delta_clad=job.delta_clad,
                         beta_clad=job.delta_clad / 80.0)
    p = wl.Problem2D("job", "fft" if job.kind == "fft2d" else "cn", xmin, xmax, dx, 0.0,
                     job.nsteps * dz, dz, job.nsteps, job.waist, guide)
    kind = pxp.FFT_SOLVER_2D if job.kind == "fft2d" else pxp.CRANK_NICHOLSON
    s = pxp.Solver(pxp.ProblemSpec(kind=kind, x=pxp.Disc(xmin, xmax, dx),
                                   z=pxp.Disc(0.0, job.nsteps * dz, dz), wavenumber=wl.K,
                                   precision=precision, device=device))
    d, b = p.material()
    s.set_material_table(d, b)
    s.set_initial_conditions(p.initial_field())
    return s


@dataclass
class RunResult:
    seconds: float
    pts_steps: float
    intensities: dict
    fields: dict = field(default_factory=dict)  # exit fields of the kept jobs

    @property
    def rate(self) -> float:
        return self.pts_steps / self.seconds


def _sync_all():
    import torch
    torch.cuda.synchronize()


def run_batched(jobs: List[Job], precision: int = pxp.FP32, max_steps: int = 100000,
                device: int = 0, keep: Optional[set] = None) -> RunResult:
    """All jobs in one Batch; returns wall time of the rounds (inputs already
    on the device) and the exit intensities and fields of the jobs listed in
    `keep`."""
    solvers = [make_solver(j, precision, device) for j in jobs]
    batch = pxp.Batch(device)
    for j, s in zip(jobs, solvers):
        if not batch.admit(s, j.nsteps):
            raise RuntimeError("memory budget exceeded")
    _sync_all()
    t0 = time.perf_counter()
    done = []
    while len(done) < len(jobs):
        batch.round(max_steps)
        done += batch.collect()
    secs = time.perf_counter() - t0
    out, fields = {}, {}
    for i, s in enumerate(solvers):
        if keep is None or i in keep:
            out[i] = s.get_intensity()
            fields[i] = s.get_last_solution()
        s.close()
    batch.close()
    return RunResult(secs, sum(j.pts_steps for j in jobs), out, fields)


def run_plain(jobs: List[Job], precision: int = pxp.FP64, device: int = 0,
              keep: Optional[set] = None) -> RunResult:
    """Each job alone, one after the other, through its own solver handle."""
    total = 0.0
    out, fields = {}, {}
    for i, j in enumerate(jobs):
        s = make_solver(j, precision, device)
        s.synchronize()
        t0 = time.perf_counter()
        s.step(j.nsteps)
        s.synchronize()
        total += time.perf_counter() - t0
        if keep is None or i in keep:
            out[i] = s.get_intensity()
            fields[i] = s.get_last_solution()
        s.close()
    return RunResult(total, sum(j.pts_steps for j in jobs), out, fields)


@dataclass
class ServeResult:
    rate: float
    jobs: int
    latencies: List[float]
    makespan: float
    pts_steps: float
    max_active: int

    @property
    def p50(self) -> float:
        return float(np.percentile(self.latencies, 50)) if self.latencies else float("nan")

    @property
    def p99(self) -> float:
        return float(np.percentile(self.latencies, 99)) if self.latencies else float("nan")

    @property
    def throughput(self) -> float:
        return self.pts_steps / self.makespan


def serve(jobs: List[Job], precision: int = pxp.FP32, round_steps: int = 200,
          hbm_budget: int = 150 * 10 ** 9, device: int = 0, results: Optional[dict] = None,
          realtime: bool = True) -> ServeResult:
    """Continuous batching.  Jobs arrive at job.arrival seconds (wall clock
    from the start); between rounds every arrived job that fits the memory
    budget is created (field and tables uploaded) and admitted; each round
    advances every admitted job by up to round_steps steps; finished jobs are
    retired, their exit intensity read back, their memory freed for the
    next admissions.  Latency = retirement time - arrival time."""
    batch = pxp.Batch(device, hbm_budget)
    pending = sorted(range(len(jobs)), key=lambda i: jobs[i].arrival)
    live = {}
    lat = []
    max_active = 0
    t0 = time.perf_counter()
    k = 0
    waiting: List[int] = []
    while k < len(pending) or waiting or live:
        now = time.perf_counter() - t0
        while k < len(pending) and (not realtime or jobs[pending[k]].arrival <= now):
            waiting.append(pending[k])
            k += 1
        still = []
        for i in waiting:
            s = make_solver(jobs[i], precision, device)
            if batch.admit(s, jobs[i].nsteps):
                live[s._h.value] = (i, s)
            else:
                s.close()
                still.append(i)
        waiting = still
        max_active = max(max_active, len(live))
        if not live:
            if k < len(pending):
                time.sleep(max(0.0, jobs[pending[k]].arrival - (time.perf_counter() - t0)))
            continue
        batch.round(round_steps)
        for s in batch.collect():
            i, _ = live.pop(s._h.value)
            t = time.perf_counter() - t0
            lat.append(t - jobs[i].arrival if realtime else t)
            inten = s.get_intensity()
            if results is not None:
                results[i] = inten
            s.close()
    makespan = time.perf_counter() - t0
    batch.close()
    span = max(makespan - (jobs[pending[0]].arrival if pending and realtime else 0.0), 1e-9)
    return ServeResult(rate=len(jobs) / max(jobs[-1].arrival, 1e-9) if jobs else 0.0,
                       jobs=len(jobs), latencies=lat, makespan=span,
                       pts_steps=sum(j.pts_steps for j in jobs), max_active=max_active)
