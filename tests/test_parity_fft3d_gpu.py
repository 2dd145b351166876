"""GPU parity of FFTSolver3D (2 transverse dims) against the CPU oracle,
through the C ABI.  FP64: <= 1e-10 relative L2 at every saved step; FP32
served mode: <= 1e-4 relative L2 of the intensity."""
import math
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_INT_TOL = 1e-4


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _int_rel(a, b):
    return np.linalg.norm(np.abs(a) ** 2 - np.abs(b) ** 2) / np.linalg.norm(np.abs(b) ** 2)


def _run_both(n, L, zmin, dz, nsteps, spheres, u0=None, save_every=1, precision=0, chunks=1,
              absorber=(0.0, 0.0)):
    import paxpro_b200 as pxp
    po.set_fft_parallel(True)
    xmin, xmax = -L / 2, L / 2
    dx = wl.step_for_nodes(xmin, xmax, n)
    zmax = zmin + nsteps * dz
    if u0 is None:
        u0 = np.ones((n, n), dtype=np.complex128, order="F")
    g = po.grid(xmin, xmax, dx, zmin, zmax, dz, wl.K)
    ref_out, ref_saves = po.fft3d_run(g, po.MaterialSpec(po.MAT_SPHERES, spheres=spheres), u0,
                                      nsteps, save_every, absorber[0], absorber[1])
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_3D, x=pxp.Disc(xmin, xmax, dx),
                           y=pxp.Disc(xmin, xmax, dx), z=pxp.Disc(zmin, zmax, dz),
                           wavenumber=wl.K, precision=precision, save_every=save_every,
                           absorber_width=absorber[0], absorber_damping=absorber[1])
    with pxp.Solver(spec) as s:
        s.set_material_spheres([pxp.Sphere(*sp) for sp in spheres])
        s.set_initial_conditions(u0)
        done = 0
        for c in range(chunks):
            k = nsteps // chunks if c < chunks - 1 else nsteps - done
            s.step(k)
            done += k
        out = s.get_last_solution()
        saves = [s.get_saved(i) for i in range(s.num_saved())]
    return out, saves, ref_out, ref_saves


def test_fft3d_fp64_spheres_and_refraction_integral():
    # spheres whose surfaces lie between sampling planes trigger the
    # refraction integral at their rims
    sph = [(50.0, -30.0, 6100.0, 180.0, 4e-5, 8e-7), (-150.0, 120.0, 12500.0, 100.0, 2e-5, 4e-7),
           (0.0, 0.0, 20000.0, 60.0, 5e-5, 1e-6)]
    out, saves, ref_out, ref_saves = _run_both(256, 1000.0, 0.0, 1000.0, 30, sph, save_every=5,
                                               chunks=3)
    assert len(saves) == 6
    assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL
    assert _rel(out, ref_out) <= FP64_TOL
    assert np.std(np.abs(out)) > 1e-4  # the spheres left a mark


@pytest.mark.parametrize("n", [64, 512, 2048])
def test_fft3d_fp64_sizes(n):
    sph = [(20.0, 10.0, 2500.0, 200.0, 3e-5, 6e-7)]
    out, saves, ref_out, ref_saves = _run_both(n, 1000.0, 0.0, 1000.0, 6, sph, save_every=2,
                                               chunks=2)
    assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL


def test_spheres_fft3d_fp64_full_size_near_a_sphere():
    p = wl.spheres_fft3d()
    # start two steps before the first sphere whose z-extent meets a sampling plane
    sph = sorted(p.spheres, key=lambda s: s[2])
    target = None
    for s in sph:
        iz = math.floor((s[2] + s[3]) / p.dz)
        if iz * p.dz > s[2] - s[3]:
            target = iz
            break
    assert target is not None
    zmin = (target - 2) * p.dz
    out, saves, ref_out, ref_saves = _run_both(4096, 2000.0, zmin, p.dz, 4, p.spheres,
                                               save_every=1)
    errs = [_rel(a, b) for a, b in zip(saves, ref_saves)]
    assert max(errs) <= FP64_TOL, errs
    assert np.std(np.abs(out)) > 0  # a sphere was crossed


def test_fft3d_absorber():
    n = 128
    L = 1000.0
    dx = wl.step_for_nodes(-L / 2, L / 2, n)
    g = po.grid(-L / 2, L / 2, dx, 0.0, 1e5, 1000.0, wl.K)
    u0 = po.gaussian_beam_3d(g, wl.WAVELENGTH, 120.0, cx=150.0, cy=-100.0)
    out, saves, ref_out, ref_saves = _run_both(n, L, 0.0, 1000.0, 20, [], u0=u0, save_every=5,
                                               absorber=(60.0, 40.0))
    assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL


def test_k1_gpu_vacuum_gaussian_closed_form():
    import paxpro_b200 as pxp
    n, L, w0, nsteps, dz = 512, 2000.0, 100.0, 100, 1000.0
    dx = wl.step_for_nodes(-L / 2, L / 2, n)
    g = po.grid(-L / 2, L / 2, dx, 0.0, 1e6, dz, wl.K)
    u0 = po.gaussian_beam_3d(g, wl.WAVELENGTH, w0)
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_3D, x=pxp.Disc(-L / 2, L / 2, dx),
                           y=pxp.Disc(-L / 2, L / 2, dx), z=pxp.Disc(0.0, 1e6, dz),
                           wavenumber=wl.K)
    with pxp.Solver(spec) as s:
        s.set_initial_conditions(u0)
        s.step(nsteps)
        out = s.get_last_solution()
    xs = -L / 2 + np.arange(n) * dx
    X, Y = np.meshgrid(xs, xs)
    z = nsteps * dz
    zr = math.pi * w0 ** 2 / wl.WAVELENGTH
    w = w0 * math.sqrt(1 + (z / zr) ** 2)
    inv_r = z / (z * z + zr * zr)
    exact = (w0 / w) * np.exp(-(X ** 2 + Y ** 2) / w ** 2) * \
        np.exp(0.5j * wl.K * (X ** 2 + Y ** 2) * inv_r - 1j * math.atan(z / zr))
    assert _rel(out, exact) < 1e-12


def test_fft3d_fp32_served_intensity_four_column_x_pass():
    # n >= 1024 runs the x pass four complex64 columns per CTA
    sph = [(15.0, -25.0, 8000.0, 220.0, 4e-5, 8e-7)]  # centre on a sampling plane
    out, saves, ref_out, ref_saves = _run_both(1024, 1000.0, 0.0, 1000.0, 40, sph,
                                               save_every=10, precision=1)
    assert max(_int_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP32_INT_TOL
    assert np.std(np.abs(out)) > 1e-4


def test_fft3d_fp32_served_intensity():
    rng = np.random.default_rng(5)
    sph = wl.random_spheres(rng, 8, -500.0, 500.0, 3.0e5)
    out, saves, ref_out, ref_saves = _run_both(512, 1000.0, 0.0, 1000.0, 300, sph,
                                               save_every=50, precision=1)
    assert max(_int_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP32_INT_TOL


@pytest.fixture
def _variant(monkeypatch):
    """Pin the FFTSolver3D launch variant for one test."""
    def pin(v):
        monkeypatch.setenv("PXP_FFT3D_VARIANT", str(v))
    return pin


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 2048])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("variant", [3, 4, 5])
def test_fft3d_register_line_kernel_every_size(n, precision, variant, _variant):
    """The register-resident line kernels -- variant 3 (8 points a thread,
    TMA-staged lines), variant 4 (16 points a thread, radix-16 passes, two
    line slots a CTA; from 512 points) and variant 5 (variant 4 with
    complex64 lines one a slot, four slots a CTA; FP64 runs variant 0 there)
    -- at every size they take, FP64 and
    FP32: spheres crossing the sampling planes (the refraction integral at
    their rims), the absorber, saves, and calls split in chunks (the
    forward-only and inverse-only passes at call ends)."""
    _variant(variant)
    sph = [(20.0, 10.0, 2500.0, 200.0, 3e-5, 6e-7), (-150.0, 120.0, 4100.0, 90.0, 2e-5, 4e-7)]
    out, saves, ref_out, ref_saves = _run_both(n, 1000.0, 0.0, 1000.0, 6, sph, save_every=2,
                                               chunks=2, precision=precision,
                                               absorber=(40.0, 30.0))
    assert len(saves) == 3
    if precision == 0:
        assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL
        assert _rel(out, ref_out) <= FP64_TOL
    else:
        assert max(_int_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP32_INT_TOL
    assert np.std(np.abs(out)) > 1e-5


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("variant", [3, 4, 5])
def test_fft3d_register_line_kernel_4096(precision, variant, _variant):
    _variant(variant)
    p = wl.spheres_fft3d()
    near = [s for s in p.spheres if s[2] + s[3] >= 86000.0 and s[2] - s[3] <= 92000.0]
    assert near  # step 44 of the workload samples a sphere
    out, saves, ref_out, ref_saves = _run_both(4096, 2000.0, 84000.0, p.dz, 4, near,
                                               save_every=2, precision=precision)
    if precision == 0:
        assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL
    else:
        assert max(_int_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP32_INT_TOL
    assert np.std(np.abs(out)) > 0


@pytest.mark.parametrize("n,precision", [(100, 0), (513, 0), (300, 1), (33, 0)])
def test_fft3d_sizes_other_than_powers_of_two(n, precision):
    """FFTSolver3D on any grid size (the reference plans FFTW for any n):
    Bluestein line transforms, spheres crossing the planes (refraction
    integral), the absorber, saves, chunked calls; FP64 within 1e-10 of the
    oracle, FP32 intensity within 1e-4."""
    po.set_threads(os.cpu_count() or 1)
    sph = [(20.0, 10.0, 2500.0, 200.0, 3e-5, 6e-7), (-150.0, 120.0, 4100.0, 90.0, 2e-5, 4e-7)]
    out, saves, ref_out, ref_saves = _run_both(n, 1000.0, 0.0, 1000.0, 6, sph, save_every=2,
                                               chunks=2, precision=precision,
                                               absorber=(40.0, 30.0))
    assert len(saves) == 3
    if precision == 0:
        assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL
        assert _rel(out, ref_out) <= FP64_TOL
    else:
        assert max(_int_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP32_INT_TOL
    assert np.std(np.abs(out)) > 1e-5


@pytest.mark.parametrize("n", [256, 1024])
def test_fft3d_fp64_joint_propagator_argument(n, monkeypatch):
    """PXP_FFT3D_JOINT_PROP=1: the x pass forms the reference's propagator
    argument fl(a * fl(kx^2 + ky^2)) and its sin/cos at every point instead
    of multiplying the x and y factor tables; every save within 1e-10 of the
    oracle as with the tables."""
    monkeypatch.setenv("PXP_FFT3D_JOINT_PROP", "1")
    sph = [(20.0, 10.0, 2500.0, 200.0, 3e-5, 6e-7), (-150.0, 120.0, 4100.0, 90.0, 2e-5, 4e-7)]
    out, saves, ref_out, ref_saves = _run_both(n, 1000.0, 0.0, 1000.0, 6, sph, save_every=2,
                                               chunks=2, precision=0)
    assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL
    assert _rel(out, ref_out) <= FP64_TOL
