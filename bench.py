"""Benchmark of the paraxial propagation step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cn4096_adi1024|waveguide_fft2d|mixed_batch|served]

Metric: grid-point * steps per second (whole job, all ranks).  A bench
"step" is one pass of the workload over its synthetic input:

  cn4096_adi1024 (default)
                  CrankNicholson Nx=4096, 8000 steps of 0.5 um  +  ADI 1024^2,
                  2000 steps of 1 um (unit plane wave, sphere R = 200 nm at
                  z = 1 mm), plain FP64; the two problems run concurrently on
                  two streams.  2.13e9 grid-point-steps per bench step.
  waveguide_fft2d FFTSolver2D Nx=2048, 4000 steps, FP64 (8.19e6 pt-steps).
  mixed_batch     mixed batch (512 2-D + 32 3-D problems), FP32 served mode in
                  one batch, against the same problems one at a time in FP64.
  served          serving: Poisson arrivals at 50..2000 jobs/s, p50/p99
                  latency and throughput, against plain FP64 one at a time.

Each rank runs its own replica (the path does not shard one field; weak
scaling).  Timing: CUDA events on the solvers' own streams, warm-up first,
L2 flushed (256 MB write) before every timed step, barrier +
synchronize around the timed region, max over ranks.

The default line also carries the served half of the metric: the mixed
batch's FP32-served rate over plain FP64 one job at a time (with the largest
relative intensity error against FP64) and the serving loop's p50/p99 job
latency at two arrival rates (`served`; --no-served skips it).

--impl reference times the reference's own solvers on all host cores, on a
bounded sample of the same workload per step: its sources compiled in place
(oracle/_ref, against stand-ins for the absent Armadillo/FFTW3/HDF5 headers),
or the oracle's restatement when that library was not built.  That arm
imports nothing from the CUDA package, so the CUDA library is never loaded
in it.

    python bench.py --case KIND N STEPS [--fp32] [--repeat R] [--flux]

runs one solver case (KIND fft2d, cn, adi or fft3d at transverse size N,
STEPS z steps per repeat; the workloads' synthetic fields and materials) and
prints the mean time per step (CUDA events on the solver's stream): the
small cases the ncu summaries under profiles/ were captured on.
`--case farfield N STEPS --pad L --angle A` times the 3-D far field of the
exit field after STEPS FFTSolver3D steps.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def _load_workloads():
    """paxpro_b200/workloads.py loaded by path: importing it through the
    package would load the CUDA library, which the CPU reference arm must
    not do (workloads.py itself needs only numpy)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "pxp_bench_workloads", os.path.join(ROOT, "paxpro_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses look their module up while defining
    spec.loader.exec_module(mod)
    return mod


wl = _load_workloads()

L2_FLUSH_BYTES = 256 << 20


def profiled_traffic(name: str):
    """DRAM bytes (read + write) per launch recorded in a profiles/ summary
    (ncu --set full capture of the same kernel and size); None if absent."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    unit = {"B": 1, "KB": 1e3, "MB": 1e6, "GB": 1e9}
    total = 0.0
    found = False
    with open(path) as f:
        for line in f:
            cells = [c.strip() for c in line.split("|")]
            if len(cells) > 2 and cells[1] in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
                tok = cells[2].split()
                v = float(tok[0])
                total += v * unit.get(tok[1], 1) if len(tok) > 1 else v
                found = True
    return total if found else None


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ------------------------------------------------------------ workloads --
class CnAdiWorkload:
    """CN (Nx = 4096, 8000 steps) + ADI (1024^2, 2000 steps), FP64."""
    name = "CrankNicholson Nx=4096 x 8000 steps + ADI 1024^2 x 2000 steps, FP64"

    def __init__(self, device: int, precision: int = 0):
        import paxpro_b200 as pxp
        self.pxp = pxp
        self.cn = wl.waveguide_cn()
        self.adi = wl.sphere_adi()
        c, a = self.cn, self.adi
        self.s_cn = pxp.Solver(pxp.ProblemSpec(
            kind=pxp.CRANK_NICHOLSON, x=pxp.Disc(c.xmin, c.xmax, c.dx),
            z=pxp.Disc(c.zmin, c.zmax, c.dz), wavenumber=wl.K, precision=precision,
            save_every=100, device=device))
        d, b = c.material()
        self.s_cn.set_material_table(d, b)
        self.s_adi = pxp.Solver(pxp.ProblemSpec(
            kind=pxp.ADI, x=pxp.Disc(a.xmin, a.xmax, a.dx), y=pxp.Disc(a.xmin, a.xmax, a.dx),
            z=pxp.Disc(a.zmin, a.zmax, a.dz), wavenumber=wl.K, precision=precision,
            save_every=100, device=device))
        self.s_adi.set_material_spheres([pxp.Sphere(*s) for s in a.spheres])
        self.u_cn = c.initial_field()
        self.u_adi = a.initial_field()
        self.pts_steps = c.nx * c.nsteps + a.nx * a.nx * a.nsteps
        self.solvers = [self.s_cn, self.s_adi]
        # per-step algorithmic bytes (2 x complex128 per point per CN step, per
        # ADI half step)
        self.adi_launches_per_step = 2 * a.nsteps
        self.adi_bytes_per_launch = 2 * 16 * a.nx * a.nx
        self.gpu_launches_per_step = 1 + 2 * a.nsteps
        self.h2d_bytes = 16 * (c.nx + a.nx * a.nx)
        self.d2h_bytes = 16 * (c.nx + a.nx * a.nx)

    def load_device_inputs(self):
        # inputs resident on the device (uploaded before the timed region)
        self.s_cn.set_initial_conditions(self.u_cn)
        self.s_adi.set_initial_conditions(self.u_adi)

    def run(self):
        self.s_cn.step(self.cn.nsteps)
        self.s_adi.step(self.adi.nsteps)

    def close(self):
        for s in self.solvers:
            s.close()


class WaveguideFft2dWorkload:
    name = "FFTSolver2D Nx=2048 x 4000 steps, FP64"

    def __init__(self, device: int, precision: int = 0):
        import paxpro_b200 as pxp
        self.pxp = pxp
        self.p = wl.waveguide_fft2d()
        p = self.p
        self.s = pxp.Solver(pxp.ProblemSpec(
            kind=pxp.FFT_SOLVER_2D, x=pxp.Disc(p.xmin, p.xmax, p.dx),
            z=pxp.Disc(p.zmin, p.zmax, p.dz), wavenumber=wl.K, precision=precision,
            save_every=100, device=device))
        d, b = p.material()
        self.s.set_material_table(d, b)
        self.u = p.initial_field()
        self.pts_steps = p.nx * p.nsteps
        self.solvers = [self.s]
        self.adi_launches_per_step = 0
        self.gpu_launches_per_step = 1
        self.h2d_bytes = 16 * p.nx
        self.d2h_bytes = 16 * p.nx

    def load_device_inputs(self):
        self.s.set_initial_conditions(self.u)

    def run(self):
        self.s.step(self.p.nsteps)

    def close(self):
        self.s.close()


WORKLOADS = {"cn4096_adi1024": CnAdiWorkload, "waveguide_fft2d": WaveguideFft2dWorkload}


def workload_pts_steps(workload: str) -> int:
    """Grid-point*steps of one pass of a timed workload."""
    if workload == "cn4096_adi1024":
        c, a = wl.waveguide_cn(), wl.sphere_adi()
        return c.nx * c.nsteps + a.nx * a.nx * a.nsteps
    p = wl.waveguide_fft2d()
    return p.nx * p.nsteps


def workload_config(workload: str, world: int) -> dict:
    """The `config` object of a timed workload; both arms print this same
    dict."""
    return {"workload": WORKLOADS[workload].name,
            "grid_pt_steps_per_step": workload_pts_steps(workload),
            "parallelism": f"replicas x{world} (one independent replica per GPU)",
            "l2": "GPU arm: flushed (256 MB write) before every timed step"}


def mixed_core(rank, world, device):
    """The mixed batch (512 2-D + 32 3-D problems) in FP32 served mode,
    one Batch per GPU, against the same problems run one at a time in plain
    FP64.  On N GPUs the one job set is split by the least-loaded scheduler
    (paxpro_b200.sharding); rates are summed grid-point*steps over the max
    elapsed time across ranks.  Every rank takes the same collective steps;
    rank 0 gets the summary, the others None."""
    import torch
    from paxpro_b200 import serving as sv
    from paxpro_b200 import sharding as sh
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import torch.distributed as dist
    all_jobs = sv.mixed_batch_jobs(seed=3)
    mine = sh.partition_jobs(all_jobs, world)[rank]
    jobs = [all_jobs[i] for i in mine]
    keep = set(range(0, len(jobs), 37))
    sv.run_batched(jobs[:40], precision=1)          # warm-up (kernels, pools)
    batched = sv.run_batched(jobs, precision=1, keep=keep)
    plain = sv.run_plain(jobs, precision=0, keep=keep)
    from paxpro_b200 import accuracy
    errs, perrs = [0.0], [0.0]
    for i in keep:
        e = accuracy.field_errors(batched.fields[i], plain.fields[i])
        errs.append(e["intensity_rel_l2"])
        perrs.append(e["phase_rms_rad"])
    dev = torch.device("cuda", device) if dist is not None else None
    b_pts, b_sec = sh.reduce_rate(batched.pts_steps, batched.seconds, dist, dev)
    p_pts, p_sec = sh.reduce_rate(plain.pts_steps, plain.seconds, dist, dev)
    _, err = sh.reduce_rate(0.0, max(errs), dist, dev)
    _, perr = sh.reduce_rate(0.0, max(perrs), dist, dev)
    if rank != 0:
        return None
    return {"served_fp32": b_pts / b_sec, "served_seconds": b_sec, "grid_pt_steps": b_pts,
            "plain_fp64": p_pts / p_sec, "plain_seconds": p_sec,
            "served_over_plain": (b_pts / b_sec) / (p_pts / p_sec),
            "max_rel_intensity_err_vs_fp64": err,
            "max_phase_rms_rad_vs_fp64": perr,
            "errors_checked_on": f"{len(keep)} of {len(jobs)} jobs per GPU"}


def run_mixed(args, rank, world, device):
    r = mixed_core(rank, world, device)
    if r is None:
        return None
    b_pts, b_sec = r["grid_pt_steps"], r["served_seconds"]
    return {
        "metric": "grid-pt*steps/s (FP32 served, batched)",
        "value": b_pts / b_sec,
        "unit": "grid-pt*steps/s",
        "n_gpus": world,
        "steps": 1,
        "warmup": 1,
        "ms_per_step": b_sec * 1e3,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "c64 storage, FP64 twiddle/factor products",
        "data": "synthetic (seeded mixed workload)",
        "config": {"workload": "mixed batch: 512 x 2-D (80% FFT, 20% CN) + 32 x 3-D FFT, one batch per GPU",
                   "grid_pt_steps": b_pts,
                   "sharding": "jobs split across GPUs, largest first to the least-loaded GPU",
                   "timing": "wall clock between device synchronisations, max over ranks"},
        "plain_fp64": {"value": r["plain_fp64"], "seconds": r["plain_seconds"]},
        "served_over_plain": r["served_over_plain"],
        "max_rel_intensity_err_vs_fp64": r["max_rel_intensity_err_vs_fp64"],
    }


def serving_core(rank, world, device, rates=(50, 100, 200, 500, 1000, 2000), window=None):
    """Serving: Poisson arrivals swept over rates; served FP32 continuous batching
    against plain FP64 one-at-a-time on the same job stream.  On N GPUs each
    GPU serves its own arrival stream at the rate (weak scaling); throughput
    is summed grid-point*steps over the max makespan across ranks.  Rank 0
    gets (rows, plain summary, window), the others None."""
    import torch
    from paxpro_b200 import serving as sv
    from paxpro_b200 import sharding as sh
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import torch.distributed as dist
    dev = torch.device("cuda", device) if dist is not None else None
    if window is None:
        window = float(os.environ.get("PXP_SERVE_WINDOW", "2.0"))
    sv.serve(sv.served_jobs(200.0, 0.1, seed=99), precision=1)  # warm-up
    rows = []
    for rate in rates:
        jobs = sv.served_jobs(float(rate), window, seed=4 + rate + 1000 * rank)
        r = sv.serve(jobs, precision=1, round_steps=200)
        pts, span = sh.reduce_rate(r.pts_steps, r.makespan, dist, dev)
        _, p99 = sh.reduce_rate(0.0, r.p99, dist, dev)
        rows.append({"rate_jobs_per_s_per_gpu": rate, "jobs": r.jobs, "p50_s": r.p50,
                     "p99_s_max_over_gpus": p99, "throughput": pts / span,
                     "max_active": r.max_active})
    jobs = sv.served_jobs(200.0, window, seed=204 + 1000 * rank)
    plain = sv.run_plain(jobs, precision=0)
    p_pts, p_sec = sh.reduce_rate(plain.pts_steps, plain.seconds, dist, dev)
    if rank != 0:
        return None
    return rows, {"value": p_pts / p_sec, "busy_seconds": p_sec, "jobs": len(jobs)}, window


def run_serving(args, rank, world, device):
    r = serving_core(rank, world, device)
    if r is None:
        return None
    rows, plain, window = r
    best = max(rows, key=lambda x: x["throughput"])
    return {
        "metric": "grid-pt*steps/s served (FP32); p50/p99 job latency",
        "value": best["throughput"],
        "unit": "grid-pt*steps/s",
        "n_gpus": world,
        "steps": len(rows),
        "warmup": 1,
        "ms_per_step": None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64 storage, FP64 twiddle/factor products",
        "data": "synthetic (seeded Poisson job stream)",
        "config": {"workload": f"served: Poisson arrivals, {window} s per rate, 80% FFT2D / 15% CN / "
                               "5% FFT3D, HBM budget 150 GB"},
        "rates": rows,
        "plain_fp64_one_at_a_time": plain,
    }


def precision_sweep(device, kind: str = "fft3d", every: int = 100):
    """The FP32 served mode against FP64 on the GPU over a whole workload:
    FFTSolver3D 4096^2 with 64 spheres, 1000 steps (kind "fft3d"), or ADI
    1024^2, 2000 steps (kind "adi"); the relative L2 intensity error and the
    intensity-weighted phase error (paxpro_b200.accuracy) of every
    `every`-th field, plus each precision's time per step (CUDA events on
    the solver's stream over steps 2 .. nsteps: the first step, which runs
    the kernel-variant tuner, is not timed; the saves are)."""
    import torch

    import paxpro_b200 as pxp
    from paxpro_b200 import accuracy
    p = wl.spheres_fft3d() if kind == "fft3d" else wl.sphere_adi()
    k = pxp.FFT_SOLVER_3D if kind == "fft3d" else pxp.ADI
    solvers, us = [], []
    for prec in (0, 1):
        s = pxp.Solver(pxp.ProblemSpec(
            kind=k, x=pxp.Disc(p.xmin, p.xmax, p.dx), y=pxp.Disc(p.xmin, p.xmax, p.dx),
            z=pxp.Disc(p.zmin, p.zmax, p.dz), wavenumber=wl.K, precision=prec,
            save_every=every, device=device))
        s.set_material_spheres([pxp.Sphere(*sp) for sp in p.spheres])
        s.set_initial_conditions(p.initial_field())
        st = torch.cuda.ExternalStream(s.stream_ptr(), device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.step(1)  # untimed: the first step runs the kernel-variant tuner
        s.synchronize()
        e0.record(st)
        s.step(p.nsteps - 1)
        e1.record(st)
        s.synchronize()
        us.append(e0.elapsed_time(e1) * 1e3 / (p.nsteps - 1))
        solvers.append(s)
    rows = []
    for i in range(solvers[0].num_saved()):
        r = accuracy.field_errors(solvers[1].get_saved(i), solvers[0].get_saved(i))
        rows.append({"step": (i + 1) * every, **{key: float(f"{v:.3e}") for key, v in r.items()}})
    for s in solvers:
        s.close()
    # FFTSolver3D: a step's two line passes each read and write the whole
    # field once (complex128: 16 B a point in FP64, complex64 in FP32); an
    # ADI half step does too (two a step)
    peak, peak_kind = measured_peaks()
    step_bytes = [4.0 * p.nx * p.nx * 16, 4.0 * p.nx * p.nx * 8]
    gbs = [b / (t * 1e-6) / 1e9 if t > 0 else 0.0 for b, t in zip(step_bytes, us)]
    return {"workload": f"{p.name}: {p.nx}^2, {p.nsteps} steps, {len(p.spheres)} spheres",
            "us_per_step_fp64": round(us[0], 2), "us_per_step_fp32": round(us[1], 2),
            "step_gbs_fp64": round(gbs[0], 1), "step_gbs_fp32": round(gbs[1], 1),
            "frac_of_hbm_fp64": round(gbs[0] / peak, 4), "frac_of_hbm_fp32": round(gbs[1] / peak, 4),
            "hbm_peak_gbs": peak, "hbm_peak_kind": peak_kind,
            "max_intensity_rel_l2": max(r["intensity_rel_l2"] for r in rows),
            "max_phase_rms_rad": max(r["phase_rms_rad"] for r in rows), "every": rows}


def served_half(rank, world, device):
    """The served half of the metric for the default line: the mixed batch
    (FP32 served over plain FP64, intensity error), the serving loop's
    p50/p99 at two arrival rates (2 s of arrivals each) and the FFTSolver3D
    precision sweep (rank 0 only; it needs no other rank)."""
    mixed = mixed_core(rank, world, device)
    srv = serving_core(rank, world, device, rates=(200, 1000), window=2.0)
    if rank != 0:
        return None
    rows, plain, window = srv
    return {"mixed_batch": mixed,
            "serving": {"window_s_per_rate": window, "rates": rows,
                        "plain_fp64_one_at_a_time_rate": plain["value"]},
            "precision_sweep": precision_sweep(device)}


# ------------------------------------------------------------- GPU arm --
def l2_resident_copy_gbs(device: int, nbytes: int, reps: int = 200) -> float:
    """Read + write bytes per second of a device-to-device copy whose source
    and destination (nbytes each) stay in L2: the memory system's rate for a
    working set the size of the ADI field and its half-step copy."""
    import torch
    src = torch.ones(nbytes // 8, dtype=torch.float64, device=device)
    dst = torch.empty_like(src)
    for _ in range(10):
        dst.copy_(src)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    e0.record()
    for _ in range(reps):
        dst.copy_(src)
    e1.record()
    torch.cuda.synchronize(device)
    return 2.0 * nbytes * reps / (e0.elapsed_time(e1) / 1e3) / 1e9


def run_ours(args, rank, world, device):
    import torch
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import torch.distributed as dist
    W = WORKLOADS[args.workload](device)
    streams = [torch.cuda.ExternalStream(s.stream_ptr(), device=device) for s in W.solvers]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)

    def one_step(timed):
        flush.zero_()
        torch.cuda.synchronize(device)
        W.load_device_inputs()
        torch.cuda.synchronize(device)
        ev0 = [torch.cuda.Event(enable_timing=True) for _ in streams]
        ev1 = [torch.cuda.Event(enable_timing=True) for _ in streams]
        for e, st in zip(ev0, streams):
            e.record(st)
        W.run()
        for e, st in zip(ev1, streams):
            e.record(st)
        torch.cuda.synchronize(device)
        # the region: from the first start to the last end
        per_stream = [ev0[0].elapsed_time(e) for e in ev1]
        return max(per_stream), [a.elapsed_time(b) for a, b in zip(ev0, ev1)]

    for _ in range(args.warmup):
        one_step(False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    times, stream_times = [], []
    with ClockSampler(device) as clk:
        for _ in range(args.steps):
            t, st = one_step(True)
            times.append(t)
            stream_times.append(st)
    torch.cuda.synchronize(device)
    if dist:
        dist.barrier()
    total_ms = sum(times)

    # end-to-end through the public API: host (pinned) inputs, H2D, steps, D2H
    pinned_in = [torch.from_numpy(np.ascontiguousarray(u.reshape(-1, order="F")).view(np.float64)).pin_memory()
                 for u in ([W.u_cn, W.u_adi] if args.workload == "cn4096_adi1024" else [W.u])]
    pinned_out = [torch.empty_like(t).pin_memory() for t in pinned_in]
    e2e_times = []
    for it in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize(device)
        ev0 = [torch.cuda.Event(enable_timing=True) for _ in streams]
        ev1 = [torch.cuda.Event(enable_timing=True) for _ in streams]
        for e, st in zip(ev0, streams):
            e.record(st)
        for s, buf in zip(W.solvers, pinned_in):
            s.set_initial_conditions_ptr(buf.data_ptr())
        W.run()
        for s, buf in zip(W.solvers, pinned_out):
            s.get_last_solution_ptr(buf.data_ptr())
        for e, st in zip(ev1, streams):
            e.record(st)
        torch.cuda.synchronize(device)
        if it >= args.warmup:
            e2e_times.append(max(ev0[0].elapsed_time(e) for e in ev1))
    e2e_ms = sum(e2e_times) / len(e2e_times)

    t_max = total_ms
    e2e_max = e2e_ms
    if dist:
        import torch.distributed as dist
        t = torch.tensor([total_ms, e2e_ms], dtype=torch.float64)
        if dist.get_backend() == "nccl":
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max, e2e_max = float(t[0]), float(t[1])
    W.close()
    if rank != 0:
        return None
    ms_per_step = t_max / args.steps
    value = world * W.pts_steps / (ms_per_step / 1e3)
    e2e_value = world * W.pts_steps / (e2e_max / 1e3)
    peak, peak_kind = measured_peaks()
    roofline = None
    if args.workload == "cn4096_adi1024":
        adi_ms = sum(st[1] for st in stream_times) / len(stream_times)
        per_launch_s = adi_ms / 1e3 / W.adi_launches_per_step
        achieved = W.adi_bytes_per_launch / per_launch_s / 1e9
        l2_copy = l2_resident_copy_gbs(device, W.adi_bytes_per_launch // 2)
        roofline = {"kernel": "adi_const_wave_kernel (FP64 vacuum half step, 1024^2, 7 systems per CTA)",
                    "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(achieved / peak, 4),
                    "peak_kind": peak_kind,
                    "traffic": profiled_traffic("adi_const_wave_kernel_1024.md"),
                    "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch "
                                      "from one ncu capture of this kernel at this size "
                                      "(profiles/adi_const_wave_kernel_1024.md; ncu flushes "
                                      "the caches before each replayed launch)",
                    "residency": "L2: the 16 MB field and its 16 MB half-step copy stay in the "
                                 "126 MB L2 across half steps, so `achieved` is effective "
                                 "bandwidth against the HBM copy peak, not an HBM-bound figure",
                    "l2_copy_gbs": round(l2_copy, 1),
                    "frac_of_l2_copy": round(achieved / l2_copy, 4),
                    "note": "algorithmic bytes 2 x 16 B per point per half step; l2_copy_gbs "
                            "= a 16 MB -> 16 MB device copy between L2-resident buffers, "
                            "timed in this run (read + write bytes per second)"}
    return {
        "metric": "grid-pt*steps/s (plain FP64)",
        "value": value,
        "unit": "grid-pt*steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded inputs with the benchmark configuration's shapes)",
        "config": workload_config(args.workload, world),
        "e2e": {"value": e2e_value, "unit": "grid-pt*steps/s",
                "h2d_bytes_per_step": W.h2d_bytes, "d2h_bytes_per_step": W.d2h_bytes},
        "gpu_launches": W.gpu_launches_per_step * args.steps,
        "roofline": roofline,
        "clocks": clk.summary(),
    }


# ------------------------------------------------------------- CPU arms --
def cpu_kind() -> str:
    """"reference" when the reference's own code is built (oracle/_ref, the
    reference's solver sources compiled in place), else "port" (the
    oracle's C++ restatement)."""
    from oracle import pyoracle as po
    return "reference" if po.refpin() is not None else "port"


def cpu_rate(workload: str, threads: int, scale: float = 1.0, kind: str = "port"):
    """A bounded sample of the workload on the host cores; returns
    (pt-steps/s extrapolated to the whole workload, description of the
    sample).  kind "reference" runs the reference's own solvers
    (ParaxialSimulation + CrankNicholson / ADI / FFTSolver2D compiled from
    its sources, oracle/_ref), "port" the oracle's restatement.  The z range
    of each sample run covers only the sampled steps (the reference's 2-D
    solvers keep every step's field)."""
    from oracle import pyoracle as po
    po.set_threads(threads)
    ref = kind == "reference"
    if workload == "cn4096_adi1024":
        c, a = wl.waveguide_cn(), wl.sphere_adi()
        n_cn = min(c.nsteps, max(20, int(800 * scale)))
        n_adi = min(a.nsteps, max(1, int(4 * scale)))
        g = po.grid(c.xmin, c.xmax, c.dx, c.zmin, c.zmin + (n_cn + 1) * c.dz, c.dz, wl.K)
        d, b = c.material()
        spec = po.MaterialSpec(po.MAT_XTABLE, delta_table=d, beta_table=b)
        t0 = time.perf_counter()
        if ref:
            po.ref_run2d(po.REF_CRANK_NICHOLSON, g, spec, c.initial_field(), n_cn, 0,
                         threads=threads)
        else:
            po.cn2d_run(g, spec, c.initial_field(), n_cn, 0)
        t_cn = time.perf_counter() - t0
        ga = po.grid(a.xmin, a.xmax, a.dx, a.zmin, a.zmin + (n_adi + 1) * a.dz, a.dz, wl.K)
        sph = po.MaterialSpec(po.MAT_SPHERES, spheres=a.spheres)
        t0 = time.perf_counter()
        if ref:
            po.ref_run3d(po.REF_ADI, ga, sph, a.initial_field(), n_adi, 0, threads=threads)
        else:
            po.adi3d_run(ga, sph, a.initial_field(), n_adi, 0)
        t_adi = time.perf_counter() - t0
        total = t_cn * c.nsteps / n_cn + t_adi * a.nsteps / n_adi
        pts = c.nx * c.nsteps + a.nx * a.nx * a.nsteps
        return pts / total, (f"CN {n_cn} of {c.nsteps} steps ({t_cn:.2f} s) + ADI {n_adi} of "
                             f"{a.nsteps} steps ({t_adi:.2f} s), extrapolated linearly")
    p = wl.waveguide_fft2d()
    n = min(p.nsteps, max(50, int(1000 * scale)))
    g = po.grid(p.xmin, p.xmax, p.dx, p.zmin, p.zmin + (n + 1) * p.dz, p.dz, wl.K)
    d, b = p.material()
    spec = po.MaterialSpec(po.MAT_XTABLE, delta_table=d, beta_table=b)
    t0 = time.perf_counter()
    if ref:
        po.ref_run2d(po.REF_FFT_SOLVER_2D, g, spec, p.initial_field(), n, 0, threads=threads)
    else:
        po.fft2d_run(g, spec, p.initial_field(), n, 0)
    t = time.perf_counter() - t0
    return p.nx * p.nsteps / (t * p.nsteps / n), f"FFTSolver2D {n} of {p.nsteps} steps ({t:.2f} s)"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args, rank, world):
    if rank != 0:
        return None
    if args.workload not in WORKLOADS:
        print(json.dumps({"impl": "reference", "unavailable": "the CPU restatement is timed on "
                          "the waveguide_fft2d and cn4096_adi1024 workloads only"}))
        return None
    threads = os.cpu_count() or 1
    kind = cpu_kind()
    rates, sample = [], ""
    for i in range(args.warmup + args.steps):
        # a few seconds of host work per step (CN 2400 + ADI 12 steps)
        r, sample = cpu_rate(args.workload, threads, scale=3.0, kind=kind)
        if i >= args.warmup:
            rates.append(r)
    value = statistics.median(rates)
    return {
        "impl": "reference",
        "metric": "grid-pt*steps/s (plain FP64)",
        "value": value,
        "unit": "grid-pt*steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(args.workload, world),
        "timing": f"wall clock of a bounded sample per step on {threads} host threads, "
                  "extrapolated to the whole workload",
        "cpu_baseline": {"value": value, "unit": "grid-pt*steps/s", "cores": threads,
                         "kind": kind, "sample": sample + f"; {cpu_model()}"},
        "e2e": {"value": value, "unit": "grid-pt*steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": ("the reference's own solver sources compiled in place (oracle/_ref) against "
                 "stand-ins for its absent third-party headers; FFTs by the oracle's FFT "
                 "where FFTW would run" if kind == "reference" else
                 "the oracle's C++ restatement of the reference path (oracle/_ref not built)"),
    }


# -------------------------------------------------- single cases (ncu) --
def case_solver(kind: str, n: int, steps: int, precision: int):
    """One solver with the workloads' synthetic inputs: the planar waveguide
    for the 2-D kinds, the sphere of the ADI workload (z starting two steps
    before it) and the 64-sphere set of the FFTSolver3D workload."""
    import paxpro_b200 as pxp
    if kind in ("fft2d", "cn"):
        p = wl.Problem2D("case", "fft" if kind == "fft2d" else "cn", -250.0, 250.0,
                         wl.step_for_nodes(-250.0, 250.0, n), 0.0, 1.0e9, 500.0, steps, 15.0,
                         wl.Waveguide())
        s = pxp.Solver(pxp.ProblemSpec(
            kind=pxp.FFT_SOLVER_2D if kind == "fft2d" else pxp.CRANK_NICHOLSON,
            x=pxp.Disc(p.xmin, p.xmax, p.dx), z=pxp.Disc(p.zmin, p.zmax, p.dz),
            wavenumber=wl.K, precision=precision))
        d, b = p.material()
        s.set_material_table(d, b)
    else:
        p = wl.sphere_adi(n=n) if kind == "adi" else wl.spheres_fft3d(n=n)
        zmin = p.zmin if kind == "fft3d" else 1.0e6 - 2 * p.dz
        s = pxp.Solver(pxp.ProblemSpec(
            kind=pxp.ADI if kind == "adi" else pxp.FFT_SOLVER_3D,
            x=pxp.Disc(p.xmin, p.xmax, p.dx), y=pxp.Disc(p.xmin, p.xmax, p.dx),
            z=pxp.Disc(zmin, 1.0e9, p.dz), wavenumber=wl.K, precision=precision))
        s.set_material_spheres([pxp.Sphere(*sp) for sp in p.spheres])
    s.set_initial_conditions(p.initial_field())
    return s


def run_case(args) -> int:
    """--case KIND N STEPS: mean time per step of one solver, CUDA events on
    its stream, min over --repeat repeats."""
    import torch
    kind, n, steps = args.case[0], int(args.case[1]), int(args.case[2])
    if kind == "farfield":
        return run_case_farfield(args, n, steps)
    if kind not in ("fft2d", "cn", "adi", "fft3d"):
        raise SystemExit(f"unknown case kind {kind}")
    s = case_solver(kind, n, steps, 1 if args.fp32 else 0)
    if args.flux:
        total = steps * max(args.repeat, 1)
        s.set_flux_windows(1, np.zeros(total, np.uint32), np.full(total, n - 1, np.uint32))
    st = torch.cuda.ExternalStream(s.stream_ptr())
    times = []
    for _ in range(max(args.repeat, 1)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.step(steps)
        e1.record(st)
        s.synchronize()
        times.append(e0.elapsed_time(e1) / steps)
    out = s.get_last_solution()
    assert np.all(np.isfinite(out))
    print(f"{kind} n={n} steps={steps} {'fp32' if args.fp32 else 'fp64'}"
          f"{' flux' if args.flux else ''}: "
          f"{min(times) * 1e3:.2f} us/step (min of {len(times)})", flush=True)
    s.close()
    return 0


def run_case_farfield(args, n: int, steps: int) -> int:
    """--case farfield N STEPS: FFTSolver3D steps, then the far field of the
    exit field minus a unit reference (pad --pad, angles -A..A) through
    pxp_farfield, CUDA-event time per call on the solver's stream."""
    import torch
    s = case_solver("fft3d", n, steps, 1 if args.fp32 else 0)
    s.step(steps)
    s.set_reference(np.ones((n, n), dtype=np.complex128))
    st = torch.cuda.ExternalStream(s.stream_ptr())
    kw = dict(pad_length=args.pad, phi_min=-args.angle, phi_max=args.angle, subtract_reference=True)
    res = s.farfield(**kw)
    times = []
    for _ in range(max(args.repeat, 1)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        res = s.farfield(**kw)
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    assert np.all(np.isfinite(res))
    print(f"farfield n={n} pad={args.pad} angle={args.angle}: result {res.shape[0]} x "
          f"{res.shape[1]}, {min(times):.3f} ms per call (min of {len(times)})", flush=True)
    s.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["mixed_batch", "served"], default="cn4096_adi1024")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-served", action="store_true",
                    help="leave the served half (mixed batch, serving p50/p99) out of the line")
    ap.add_argument("--case", nargs=3, metavar=("KIND", "N", "STEPS"),
                    help="time one solver case (fft2d, cn, adi, fft3d, farfield) and exit")
    ap.add_argument("--fp32", action="store_true", help="--case: FP32 served mode")
    ap.add_argument("--repeat", type=int, default=1, help="--case: repeats (min reported)")
    ap.add_argument("--flux", action="store_true", help="--case: per-step flux windows")
    ap.add_argument("--pad", type=int, default=32768, help="--case farfield: pad length")
    ap.add_argument("--angle", type=float, default=0.05, help="--case farfield: max angle (deg)")
    args = ap.parse_args()
    if args.case:
        sys.exit(run_case(args))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload == "mixed_batch":
        out = run_mixed(args, rank, world, local)
    elif args.workload == "served":
        out = run_serving(args, rank, world, local)
    else:
        out = run_ours(args, rank, world, local)
    if args.workload == "cn4096_adi1024" and not args.no_served:
        served = served_half(rank, world, local)
        if out is not None:
            out["served"] = served
    if out is not None and not args.no_cpu_baseline and args.workload in ("waveguide_fft2d", "cn4096_adi1024"):
        # about 10 s of single-thread work (CN 8000 + ADI 32 steps)
        kind = cpu_kind()
        rate, sample = cpu_rate(args.workload, 1, scale=8.0 if kind == "reference" else 15.0,
                                kind=kind)
        out["cpu_baseline"] = {"value": rate, "unit": "grid-pt*steps/s", "cores": 1,
                               "kind": kind, "sample": sample + f"; {cpu_model()}"}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
