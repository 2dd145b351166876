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


@pytest.mark.parametrize("kind,n", [("fft", 128), ("adi", 128), ("adi", 129)])
def test_generic_scattering_example(kind, n):
    """GenericScattering: the vacuum reference run (three steps), the run
    through the sphere and the far field of the difference, resized to the
    export dimensions, against the oracle."""
    from oracle import farfield as off
    exe = build("scattering3d")
    steps, pad, ang, exp = 6, 1024, 0.05, 64
    out = os.path.join(OUT, f"gs_{kind}_{n}.bin")
    r = subprocess.run([exe, kind, str(n), str(steps), str(pad), str(ang), str(exp), out],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.float64)
    N, rows, cols = int(data[0]), int(data[1]), int(data[2])
    c = data[3:3 + 6 * N * N].view(np.complex128)
    u0, ref, ex = (c[k * N * N:(k + 1) * N * N].reshape((N, N), order="F") for k in range(3))
    ff = data[3 + 6 * N * N:].reshape((rows, cols), order="F")
    K = 2.0 * math.pi / 0.1569
    dx = _dx(n, 1000.0)
    g0 = po.grid(-500.0, 500.0, dx, -300.0, 300.0, 200.0, K)
    g1 = po.grid(-500.0, 500.0, dx, -300.0, 300.0, 600.0 / steps, K)
    assert _rel(u0, po.gaussian_beam_3d(g0, 0.1569, 300.0)) <= 1e-13
    sphere = po.MaterialSpec(po.MAT_SPHERES, spheres=[(20.0, -10.0, 0.0, 200.0, 8.9e-6, 7e-7)])
    if kind == "fft":
        ref_o, _ = po.fft3d_run(g0, po.MaterialSpec(), u0, 3, 0)
        ex_o, _ = po.fft3d_run(g1, sphere, u0, steps, 0)
    else:
        ref_o, _ = po.adi3d_run(g0, po.MaterialSpec(), u0, 3, 0, True)
        ex_o, _ = po.adi3d_run(g1, sphere, u0, steps, 0, True)
    assert _rel(ref, ref_o) <= TOL
    assert _rel(ex, ex_o) <= TOL
    ff_o = off.farfield_3d(ex, pad, -ang, ang, K, dx, dx, reference=ref, export_rows=exp,
                           export_cols=exp)
    assert ff.shape == ff_o.shape == (exp, exp)
    assert _rel(ff, ff_o) <= TOL


@pytest.mark.parametrize("kind,smoothed", [("cn", 0), ("fft", 0), ("cn", 1)])
def test_curved_waveguide_transmittivity(kind, smoothed):
    """CurvedWaveGuideFD::solve with post::Transmittivity: the transmission
    the step kernels integrate equals Transmittivity::compute
    (src/transmittivity.cpp:30-83) evaluated on the saved fields."""
    exe = build("curved2d")
    n, steps = 1024, 150
    out = os.path.join(OUT, f"cw_{kind}_{smoothed}.bin")
    r = subprocess.run([exe, kind, str(n), str(steps), str(smoothed), out], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.float64)
    nx, nz, i0 = int(data[0]), int(data[1]), data[2]
    t = data[3:3 + nz - 1]
    sol = data[3 + nz - 1:].view(np.complex128).reshape((nx, nz), order="F")
    xmin, xmax, R, width, dz = -400.0, 200.0, 40e6, 100.0, 500.0
    dx = wl.step_for_nodes(xmin, xmax, n)

    def closest(x):
        return int((x - xmin) / dx)

    def integral(u, a, b):
        total = abs(u[a]) ** 2 + abs(u[b]) ** 2
        for i in range(a + 1, b):
            total += 2.0 * abs(u[i]) ** 2
        step = ((xmin + b * dx) - (xmin + a * dx)) / (b - a)
        return total * step * 0.5

    I0 = integral(sol[:, 1], closest(0.0), closest(width))
    want = []
    for k in range(1, nz):
        z = 0.0 + k * dz
        start = -0.5 * z * z / R
        want.append(integral(sol[:, k], closest(start), closest(start + width)) / I0)
    assert i0 == pytest.approx(I0, rel=1e-12)
    np.testing.assert_allclose(t, np.array(want), rtol=1e-12, atol=0)
    assert 0.0 < t[-1] < 1.0


@pytest.mark.parametrize("prop", ["fft", "adi"])
def test_reference_sphere_example_with_a_user_material_function(prop):
    """The reference's Examples/sphere.cpp through the B200 API: a user
    MaterialFunction subclass (not a type the device evaluates), sampled on
    the host at the planes the solver samples, 513 transverse nodes
    (FFTSolver3D: Bluestein line transforms, the example's default
    propagator; ADI: the padded general kernel), 256 steps,
    GenericScattering's vacuum reference run and far field.  Exit fields
    against the oracle with the same sphere (1e-10), the far field against
    the numpy far field of those fields."""
    from oracle import farfield as off
    exe = build("example_sphere")
    out = os.path.join(OUT, f"example_sphere_{prop}.bin")
    r = subprocess.run([exe, out, prop], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.float64)
    N, rows, cols = int(data[0]), int(data[1]), int(data[2])
    assert N == 513
    c = data[3:3 + 4 * N * N].view(np.complex128)
    ref, ex = (c[k * N * N:(k + 1) * N * N].reshape((N, N), order="F") for k in range(2))
    ff = data[3 + 4 * N * N:].reshape((rows, cols), order="F")
    K = 2.0 * math.pi / 0.1569
    dx = 1500.0 / 512
    g0 = po.grid(-750.0, 750.0, dx, -525.0, 525.0, 1050.0 / 3.0, K)
    g1 = po.grid(-750.0, 750.0, dx, -525.0, 525.0, 1050.0 / 256, K)
    u0 = po.gaussian_beam_3d(g0, 0.1569, 200000.0)
    sphere = po.MaterialSpec(po.MAT_SPHERES, spheres=[(0.0, 0.0, 0.0, 500.0, 8.9e-6, 7e-7)])
    if prop == "adi":
        ref_o, _ = po.adi3d_run(g0, po.MaterialSpec(), u0, 3, 0, True)
        ex_o, _ = po.adi3d_run(g1, sphere, u0, 256, 0, True)
    else:
        po.set_fft_parallel(True)
        po.set_threads(os.cpu_count() or 1)
        ref_o, _ = po.fft3d_run(g0, po.MaterialSpec(), u0, 3, 0)
        ex_o, _ = po.fft3d_run(g1, sphere, u0, 256, 0)
    assert _rel(ref, ref_o) <= TOL
    assert _rel(ex, ex_o) <= TOL
    assert np.std(np.abs(ex)) > 1e-3  # the sphere left its mark
    ff_o = off.farfield_3d(ex, 1024, -0.05, 0.05, K, dx, dx, reference=ref, export_rows=512,
                           export_cols=512)
    assert ff.shape == ff_o.shape
    assert _rel(ff, ff_o) <= TOL
