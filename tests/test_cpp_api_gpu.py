"""GPU runs of the C++ solver API examples (tests/cpp) against the oracle:
the reference's usage pattern (material function, Gaussian beam or plane
wave, ParaxialSimulation::setSolver / setBoundaryConditions / solve,
getLastSolution / getSolution) produces the oracle's fields within the FP64
tolerance (1e-10 relative L2)."""
import math
import os
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import workloads as wl
from tests.cpp_build import OUT, build

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _dx(n, L):
    return wl.step_for_nodes(-L / 2, L / 2, n)


@pytest.mark.parametrize("kind,transparent,zvary", [("fft", 0, 0), ("fft", 0, 1), ("cn", 0, 0),
                                                     ("cn", 1, 0), ("cn", 0, 1)])
def test_waveguide2d_example(kind, transparent, zvary):
    exe = build("waveguide2d")
    n, steps = 512, 300
    out = os.path.join(OUT, f"wg_{kind}_{transparent}_{zvary}.bin")
    r = subprocess.run([exe, kind, str(n), str(steps), out, str(transparent), str(zvary)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.complex128)
    last, mid, first = data[:n], data[n:2 * n], data[2 * n:3 * n]
    dz = 500.0 if kind == "cn" else 1000.0
    g = po.grid(-250.0, 250.0, _dx(n, 500.0), 0.0, steps * dz, dz, wl.K)
    spec = po.MaterialSpec(po.MAT_WAVEGUIDE, core_half_width=25.0, delta_clad=7.5e-6,
                           beta_clad=1e-7, ramp_points=25, ramp_beta=1e-4, n_transverse=n)
    u0 = po.gaussian_beam_2d(g, 0.1, 15.0, center=40.0 if kind == "cn" else 0.0)
    assert np.array_equal(first, u0)
    run = po.fft2d_run if kind == "fft" else po.cn2d_run
    extra = {} if kind == "fft" else {"transparent": bool(transparent)}
    ref_last, ref_saves = run(g, spec, u0, steps, 1, **extra)
    assert _rel(last, ref_last) <= TOL
    assert _rel(mid, ref_saves[steps // 2 - 1]) <= TOL


@pytest.mark.parametrize("kind", ["fft3d", "adi"])
def test_sphere3d_example(kind):
    exe = build("sphere3d")
    n, steps, ratio = 128, 10, 5
    out = os.path.join(OUT, f"sp_{kind}.bin")
    r = subprocess.run([exe, kind, str(n), str(steps), str(ratio), out], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.complex128)
    last = data[:n * n].reshape((n, n), order="F")
    slice1 = data[n * n:2 * n * n].reshape((n, n), order="F")
    g = po.grid(-500.0, 500.0, _dx(n, 1000.0), 0.0, steps * 1000.0, 1000.0, wl.K)
    sph = [(40.0, -30.0, 3000.0, 150.0, 4.5e-5, 9e-7), (-120.0, 90.0, 6500.0, 100.0, 2e-5, 4e-7)]
    spec = po.MaterialSpec(po.MAT_SPHERES, spheres=sph)
    u0 = np.ones((n, n), dtype=np.complex128, order="F")
    if kind == "fft3d":
        ref_last, ref_saves = po.fft3d_run(g, spec, u0, steps, ratio)
    else:
        ref_last, ref_saves = po.adi3d_run(g, spec, u0, steps, ratio, False)
    assert _rel(last, ref_last) <= TOL
    assert _rel(slice1, ref_saves[0]) <= TOL


@pytest.mark.parametrize("kind", ["fft3d", "adi"])
def test_csg3d_example(kind):
    """CSGMaterial built from geom:: shapes in C++ propagates to the oracle's
    fields for the same geometry built by the Python classes."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from csg_geometry import geometry
    from paxpro_b200 import csg
    exe = build("csg3d")
    n, steps = 128, 7
    out = os.path.join(OUT, f"csg_{kind}.bin")
    r = subprocess.run([exe, kind, str(n), str(steps), out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.complex128)
    last = data[:n * n].reshape((n, n), order="F")
    slice1 = data[n * n:2 * n * n].reshape((n, n), order="F")
    g = po.grid(-500.0, 500.0, _dx(n, 1000.0), 0.0, steps * 1000.0, 1000.0, wl.K)
    spec = po.MaterialSpec(po.MAT_CSG, csg=csg.flatten(geometry()))
    u0 = np.ones((n, n), dtype=np.complex128, order="F")
    if kind == "fft3d":
        ref_last, ref_saves = po.fft3d_run(g, spec, u0, steps, 1)
    else:
        ref_last, ref_saves = po.adi3d_run(g, spec, u0, steps, 1, False)
    assert _rel(last, ref_last) <= TOL
    assert _rel(slice1, ref_saves[0]) <= TOL
    assert np.std(np.abs(last)) > 1e-4
