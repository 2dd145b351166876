"""The workloads as they are timed, on the GPU.

* ADI, FP64, 1024^2 over all 2000 steps of the sphere workload (the bench's
  ADI problem), every 100th field against the oracle: <= 1e-10 relative L2.
  The vacuum half steps run the fast path (host factor tables, scans), whose
  rounding differs from the reference's Thomas sweep at the last bits; this
  shows that the difference does not grow past the tolerance over the run.
* FFTSolver3D, FP64, 4096^2 with the workload's 64 spheres over 110 steps
  (steps 250-359 of its 1000: four spheres sampled, their refraction-integral
  rims included), every 22nd field against the oracle.  The GPU gets all 64
  spheres; the oracle only those whose z extent reaches the run's planes
  (the others contain no sampled point, so the medium is the same) to keep
  its CPU time down.
* The precision sweep: FFTSolver3D 4096^2, 1000 steps, FP32 served mode
  against the FP64 run (itself parity-tested above): relative L2 intensity
  error <= 1e-4 and the intensity-weighted phase error at every 100th step.
* ADI FP32 at 1024^2 over the 2000 steps against the FP64 run, likewise.

The oracle uses every host core (its transforms and the ADI systems run in
parallel; results do not depend on the thread count)."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import accuracy
from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_INT_TOL = 1e-4
FP32_PHASE_TOL = 1e-3  # radians, intensity-weighted RMS


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _solver(pxp, kind, p, zmin, nsteps, precision, save_every, spheres):
    spec = pxp.ProblemSpec(kind=kind, x=pxp.Disc(p.xmin, p.xmax, p.dx),
                           y=pxp.Disc(p.xmin, p.xmax, p.dx),
                           z=pxp.Disc(zmin, zmin + nsteps * p.dz, p.dz), wavenumber=wl.K,
                           precision=precision, save_every=save_every)
    s = pxp.Solver(spec)
    s.set_material_spheres([pxp.Sphere(*sp) for sp in spheres])
    s.set_initial_conditions(p.initial_field())
    return s


def _cull(spheres, zlo, zhi):
    """Spheres whose z extent reaches [zlo, zhi]."""
    return [s for s in spheres if s[2] + s[3] >= zlo and s[2] - s[3] <= zhi]


@pytest.fixture(scope="module", autouse=True)
def _oracle_threads():
    po.set_threads(os.cpu_count() or 1)
    po.set_fft_parallel(True)
    yield
    po.set_fft_parallel(False)


def test_sphere_adi_fp64_all_2000_steps_against_oracle():
    import paxpro_b200 as pxp
    p = wl.sphere_adi()
    with _solver(pxp, pxp.ADI, p, p.zmin, p.nsteps, 0, 100, p.spheres) as s:
        s.step(p.nsteps)
        saves = [s.get_saved(i) for i in range(s.num_saved())]
    g = po.grid(p.xmin, p.xmax, p.dx, p.zmin, p.zmax, p.dz, wl.K)
    _, ref = po.adi3d_run(g, po.MaterialSpec(po.MAT_SPHERES, spheres=p.spheres),
                          p.initial_field(), p.nsteps, 100)
    assert len(saves) == len(ref) == 20
    errs = [_rel(a, b) for a, b in zip(saves, ref)]
    assert max(errs) <= FP64_TOL, errs
    assert np.std(np.abs(saves[-1])) > 1e-3  # the sphere at z = 1 mm left its mark


def test_spheres_fft3d_fp64_110_steps_at_4096_against_oracle():
    import paxpro_b200 as pxp
    p = wl.spheres_fft3d()
    first, nsteps, every = 250, 110, 22
    zmin = p.zmin + (first - 1) * p.dz
    zmax = zmin + nsteps * p.dz
    near = _cull(p.spheres, zmin, zmax)
    assert len(near) >= 4
    with _solver(pxp, pxp.FFT_SOLVER_3D, p, zmin, nsteps, 0, every, p.spheres) as s:
        s.step(nsteps)
        saves = [s.get_saved(i) for i in range(s.num_saved())]
    g = po.grid(p.xmin, p.xmax, p.dx, zmin, zmax, p.dz, wl.K)
    _, ref = po.fft3d_run(g, po.MaterialSpec(po.MAT_SPHERES, spheres=near), p.initial_field(),
                          nsteps, every)
    assert len(saves) == len(ref) == nsteps // every
    errs = [_rel(a, b) for a, b in zip(saves, ref)]
    assert max(errs) <= FP64_TOL, errs
    assert np.std(np.abs(saves[-1])) > 1e-4  # spheres were crossed


def _precision_sweep(kind, p, every):
    """FP32 against FP64 on the GPU at every `every` steps: per save the
    intensity and phase errors."""
    import paxpro_b200 as pxp
    rows = []
    with _solver(pxp, kind, p, p.zmin, p.nsteps, 0, every, p.spheres) as s64, \
            _solver(pxp, kind, p, p.zmin, p.nsteps, 1, every, p.spheres) as s32:
        s64.step(p.nsteps)
        s32.step(p.nsteps)
        for i in range(s64.num_saved()):
            rows.append(accuracy.field_errors(s32.get_saved(i), s64.get_saved(i)))
    return rows


def test_spheres_fft3d_precision_sweep_fp32_against_fp64():
    import paxpro_b200 as pxp
    rows = _precision_sweep(pxp.FFT_SOLVER_3D, wl.spheres_fft3d(), 100)
    assert len(rows) == 10
    assert max(r["intensity_rel_l2"] for r in rows) <= FP32_INT_TOL, rows
    assert max(r["phase_rms_rad"] for r in rows) <= FP32_PHASE_TOL, rows


def test_sphere_adi_fp32_against_fp64_all_2000_steps():
    import paxpro_b200 as pxp
    rows = _precision_sweep(pxp.ADI, wl.sphere_adi(), 100)
    assert len(rows) == 20
    assert max(r["intensity_rel_l2"] for r in rows) <= FP32_INT_TOL, rows
    assert max(r["phase_rms_rad"] for r in rows) <= FP32_PHASE_TOL, rows
