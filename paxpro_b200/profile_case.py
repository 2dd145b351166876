"""Run one solver case on the GPU, for profiling and quick timing.

    python -m paxpro_b200.profile_case KIND N STEPS [--fp32] [--repeat R]

KIND is fft2d, cn, adi or fft3d; N the transverse size; STEPS the number of
z steps per repeat.  Inputs are the benchmark workloads' synthetic fields and
materials (planar waveguide for the 2-D kinds, the config-1 sphere for ADI,
the config-2 sphere set for FFT3D).  Prints the mean time per step measured
with CUDA events on the solver's stream.

    python -m paxpro_b200.profile_case farfield N STEPS --pad L --angle A

runs STEPS FFTSolver3D steps of the config-2 workload at size N, then times
the 3-D far field of the exit field (pad length L, angles -A..A degrees,
the subtraction of a reference field included) through pxp_farfield:
CUDA-event time on the solver's stream around the call (the transforms, the
reference subtraction and the copy of the result to the host).
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys

import numpy as np

import paxpro_b200 as pxp
from paxpro_b200 import workloads as wl


def make(kind: str, n: int, steps: int, precision: int):
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
        u0 = p.initial_field()
    else:
        p = wl.sphere_adi(n=n) if kind == "adi" else wl.spheres_fft3d(n=n)
        zmin = p.zmin if kind == "fft3d" else 1.0e6 - 2 * p.dz
        s = pxp.Solver(pxp.ProblemSpec(
            kind=pxp.ADI if kind == "adi" else pxp.FFT_SOLVER_3D,
            x=pxp.Disc(p.xmin, p.xmax, p.dx), y=pxp.Disc(p.xmin, p.xmax, p.dx),
            z=pxp.Disc(zmin, 1.0e9, p.dz), wavenumber=wl.K, precision=precision))
        s.set_material_spheres([pxp.Sphere(*sp) for sp in p.spheres])
        u0 = p.initial_field()
    s.set_initial_conditions(u0)
    return s


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("kind", choices=["fft2d", "cn", "adi", "fft3d", "farfield"])
    ap.add_argument("n", type=int)
    ap.add_argument("steps", type=int)
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--flux", action="store_true",
                    help="2-D kinds: per-step flux windows over the whole line (Transmittivity)")
    ap.add_argument("--pad", type=int, default=32768)
    ap.add_argument("--angle", type=float, default=0.05)
    a = ap.parse_args(argv)
    if a.kind == "farfield":
        return farfield(a)
    s = make(a.kind, a.n, a.steps, 1 if a.fp32 else 0)
    if a.flux:
        total = a.steps * max(a.repeat, 1)
        s.set_flux_windows(1, np.zeros(total, np.uint32), np.full(total, a.n - 1, np.uint32))
    import torch
    st = torch.cuda.ExternalStream(s.stream_ptr())
    times = []
    for _ in range(a.repeat):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.step(a.steps)
        e1.record(st)
        s.synchronize()
        times.append(e0.elapsed_time(e1) / a.steps)
    out = s.get_last_solution()
    assert np.all(np.isfinite(out))
    print(f"{a.kind} n={a.n} steps={a.steps} {'fp32' if a.fp32 else 'fp64'}"
          f"{' flux' if a.flux else ''}: "
          f"{min(times) * 1e3:.2f} us/step (min of {a.repeat})")
    s.close()
    return 0


def farfield(a) -> int:
    import torch
    s = make("fft3d", a.n, a.steps, 1 if a.fp32 else 0)
    s.step(a.steps)
    s.set_reference(np.ones((a.n, a.n), dtype=np.complex128))
    st = torch.cuda.ExternalStream(s.stream_ptr())
    res = s.farfield(pad_length=a.pad, phi_min=-a.angle, phi_max=a.angle, subtract_reference=True)
    times = []
    for _ in range(max(a.repeat, 1)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        res = s.farfield(pad_length=a.pad, phi_min=-a.angle, phi_max=a.angle,
                         subtract_reference=True)
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    assert np.all(np.isfinite(res))
    print(f"farfield n={a.n} pad={a.pad} angle={a.angle}: result {res.shape[0]} x {res.shape[1]}, "
          f"{min(times):.3f} ms per call (min of {len(times)})")
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
