"""Saved slices of the 3-D solvers with a transverse downsampling ratio:
block averages as Solver3D::copyCurrentSolution stores them
(src/solver3D.cpp:94-112), computed on the device, against the oracle's
full saves reduced by the oracle's restatement of the same average.  Ratio 3
on 256 points gives 85 x 85 slices with non-integer block bounds."""
import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _int_rel(a, b):
    return np.linalg.norm(np.abs(a) ** 2 - np.abs(b) ** 2) / np.linalg.norm(np.abs(b) ** 2)


def _run(kind, n, ratio, nsteps, precision=0):
    import paxpro_b200 as pxp
    po.set_fft_parallel(True)
    L, dz = 1000.0, 1000.0
    xmin, xmax = -L / 2, L / 2
    dx = wl.step_for_nodes(xmin, xmax, n)
    sph = [(20.0, -30.0, 3000.0, 160.0, 4e-5, 2e-6)]
    g = po.grid(xmin, xmax, dx, 0.0, nsteps * dz, dz, wl.K)
    mat = po.MaterialSpec(po.MAT_SPHERES, spheres=sph)
    u0 = np.ones((n, n), dtype=np.complex128, order="F")
    if kind == "fft3d":
        _, ref_saves = po.fft3d_run(g, mat, u0, nsteps, 2)
    else:
        _, ref_saves = po.adi3d_run(g, mat, u0, nsteps, 2)
    ref = [po.block_average(f, ratio) for f in ref_saves]
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_3D if kind == "fft3d" else pxp.ADI,
                           x=pxp.Disc(xmin, xmax, dx, ratio), y=pxp.Disc(xmin, xmax, dx, ratio),
                           z=pxp.Disc(0.0, nsteps * dz, dz), wavenumber=wl.K,
                           precision=precision, save_every=2)
    with pxp.Solver(spec) as s:
        s.set_material_spheres([pxp.Sphere(*sp) for sp in sph])
        s.set_initial_conditions(u0)
        s.step(nsteps)
        got = [s.get_saved(i) for i in range(s.num_saved())]
    return got, ref


@pytest.mark.parametrize("kind", ["fft3d", "adi"])
@pytest.mark.parametrize("ratio", [2, 3])
def test_downsampled_saves_fp64(kind, ratio):
    got, ref = _run(kind, 256, ratio, 8)
    m = 256 // ratio
    assert len(got) == len(ref) == 4
    assert all(g.shape == (m, m) for g in got)
    errs = [_rel(a, b) for a, b in zip(got, ref)]
    assert max(errs) <= 1e-10, errs
    assert np.std(np.abs(got[-1])) > 1e-5  # the sphere left a mark


def test_downsampled_saves_fp32_served():
    got, ref = _run("fft3d", 512, 4, 8, precision=1)
    assert all(g.shape == (128, 128) for g in got)
    assert max(_int_rel(a, b) for a, b in zip(got, ref)) <= 1e-4
