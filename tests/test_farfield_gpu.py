"""post::FarField on the device (pxp_farfield) against the oracle
(oracle/farfield.py) on the same exit field: FP64 <= 1e-10 relative L2.
Covers the pruned padded transform and the direct DFT (power-of-two and
other pad lengths, each path pinned), wide and narrow angular windows,
2-D pad values, 3-D zero and constant padding, reference subtraction from a
host array and from another handle, resizeMatrix and FP32 fields."""
import os

import numpy as np
import pytest

from oracle import farfield as off
from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(params=["auto", "direct", "pruned"])
def path(request, monkeypatch):
    if request.param != "auto":
        monkeypatch.setenv("PXP_FARFIELD_PATH", request.param)
    return request.param


def _solver2d(kind, n, precision=0, steps=40):
    import paxpro_b200 as pxp
    L = 500.0
    dx = wl.step_for_nodes(-L / 2, L / 2, n)
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D if kind == "fft" else pxp.CRANK_NICHOLSON,
                           x=pxp.Disc(-L / 2, L / 2, dx), z=pxp.Disc(0.0, steps * 500.0, 500.0),
                           wavenumber=wl.K, precision=precision)
    s = pxp.Solver(spec)
    x = -L / 2 + dx * np.arange(n)
    s.set_material_table(np.where(np.abs(x) < 25.0, 0.0, 7.5e-6), np.full(n, 1e-8))
    s.set_initial_conditions(np.exp(-x ** 2 / 15.0 ** 2).astype(np.complex128))
    s.step(steps)
    return s, dx


def _solver3d(kind, n, precision=0, steps=5, material=True):
    import paxpro_b200 as pxp
    xmin, xmax = -500.0, 500.0
    dx = wl.step_for_nodes(xmin, xmax, n)
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_3D if kind == "fft3d" else pxp.ADI,
                           x=pxp.Disc(xmin, xmax, dx), y=pxp.Disc(xmin, xmax, dx),
                           z=pxp.Disc(0.0, steps * 1000.0, 1000.0), wavenumber=wl.K,
                           precision=precision)
    s = pxp.Solver(spec)
    if material:
        s.set_material_spheres([pxp.Sphere(30.0, -40.0, 3000.0, 200.0, 4e-5, 2e-6)])
    s.set_initial_conditions(np.ones((n, n), dtype=np.complex128, order="F"))
    s.step(steps)
    return s, dx


@pytest.mark.parametrize("kind,n,pad,phi", [("fft", 512, 4096, 90.0), ("fft", 512, 4096, 0.02),
                                            ("fft", 512, 0, 90.0), ("cn", 256, 1000, 90.0),
                                            ("cn", 256, 1024, 0.05), ("fft", 256, 32768, 0.002)])
def test_farfield_2d(kind, n, pad, phi, path):
    s, dx = _solver2d(kind, n)
    with s:
        u = s.get_last_solution()
        for pv in (0.0, 0.25 - 0.1j):
            got = s.farfield(pad_length=pad, phi_min=-phi, phi_max=phi, pad_value=pv)
            want = off.farfield_2d(u, pad, -phi, phi, wl.K, dx, pad_value=pv)
            assert got.shape == want.shape
            assert _rel(got, want) <= TOL


@pytest.mark.parametrize("kind,n,pad,phi", [("fft3d", 128, 1024, 90.0), ("fft3d", 128, 1000, 90.0),
                                            ("adi", 128, 0, 90.0), ("fft3d", 256, 2048, 0.03)])
def test_farfield_3d(kind, n, pad, phi, path):
    s, dx = _solver3d(kind, n)
    with s:
        u = s.get_last_solution()
        got = s.farfield(pad_length=pad, phi_min=-phi, phi_max=phi)
        want = off.farfield_3d(u, pad, -phi, phi, wl.K, dx, dx)
        assert got.shape == want.shape
        assert _rel(got, want) <= TOL
        got = s.farfield(pad_length=pad, phi_min=-phi, phi_max=phi, padding=off.PAD_CONSTANT)
        want = off.farfield_3d(u, pad, -phi, phi, wl.K, dx, dx, padding=off.PAD_CONSTANT)
        assert _rel(got, want) <= TOL


def test_farfield_3d_reference_runs_and_resize():
    import paxpro_b200 as pxp
    n, pad = 128, 1024
    s, dx = _solver3d("fft3d", n)
    r, _ = _solver3d("fft3d", n, material=False)
    with s, r:
        u, ref = s.get_last_solution(), r.get_last_solution()
        assert _rel(u, ref) > 1e-3                # the sphere scattered
        want = off.farfield_3d(u, pad, -90.0, 90.0, wl.K, dx, dx, reference=ref)
        s.set_reference(r)                     # device copy from the other handle
        got = s.farfield(pad_length=pad, subtract_reference=True)
        assert _rel(got, want) <= TOL
        s.set_reference(ref)                   # host array
        got = s.farfield(pad_length=pad, subtract_reference=True)
        assert _rel(got, want) <= TOL
        want_small = off.farfield_3d(u, pad, -90.0, 90.0, wl.K, dx, dx, reference=ref,
                                     export_rows=100, export_cols=90)
        got_small = s.farfield(pad_length=pad, subtract_reference=True, export_dims=(100, 90))
        assert got_small.shape == (100, 90)
        assert _rel(got_small, want_small) <= TOL
        s.set_reference(None)
        with pytest.raises(pxp.PxpError):
            s.farfield(pad_length=pad, subtract_reference=True)


def test_farfield_fp32_field_and_errors():
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi
    s, dx = _solver3d("fft3d", 128, precision=1)
    with s:
        u = s.get_last_solution()           # complex64 values widened
        got = s.farfield(pad_length=512)
        want = off.farfield_3d(u, 512, -90.0, 90.0, wl.K, dx, dx)
        assert _rel(got, want) <= TOL
        with pytest.raises(pxp.PxpError):
            s.farfield(padding=_capi.PAD_LINEAR_FIT)
        with pytest.raises(pxp.PxpError):
            s.farfield(phi_min=10.0, phi_max=-10.0)


@pytest.mark.parametrize("propagator", ["fft", "adi"])
def test_python_generic_scattering(propagator, tmp_path):
    """paxpro_b200.scattering.GenericScattering: the reference run, the sample
    run and the far field against the oracle on the same fields."""
    import paxpro_b200 as pxp
    from oracle import pyoracle as po
    from paxpro_b200.scattering import GenericScattering
    n, steps = 128, 6
    dx = wl.step_for_nodes(-500.0, 500.0, n)
    with GenericScattering("sphere") as gs:
        gs.setBeamWaist(300.0)
        gs.setMaxScatteringAngle(0.05)
        gs.xmin = gs.ymin = -500.0
        gs.xmax = gs.ymax = 500.0
        gs.zmin, gs.zmax = -300.0, 300.0
        gs.dx = gs.dy = dx
        gs.dz = 600.0 / steps
        gs.FFTPadLength = 1024
        gs.exportNx = gs.exportNy = 64
        gs.propagator = propagator
        gs.setMaterial([pxp.Sphere(20.0, -10.0, 0.0, 200.0, 8.9e-6, 7e-7)])
        gs.solve()
        ff = gs.getFarField()
        K = 2.0 * np.pi / 0.1569
        g0 = po.grid(-500.0, 500.0, dx, -300.0, 300.0, 200.0, K)
        g1 = po.grid(-500.0, 500.0, dx, -300.0, 300.0, 100.0, K)
        u0 = po.gaussian_beam_3d(g0, 0.1569, 300.0)
        assert _rel(gs._initial(), u0) <= 1e-13
        sph = po.MaterialSpec(po.MAT_SPHERES, spheres=[(20.0, -10.0, 0.0, 200.0, 8.9e-6, 7e-7)])
        if propagator == "fft":
            ref_o, _ = po.fft3d_run(g0, po.MaterialSpec(), u0, 3, 0)
            ex_o, _ = po.fft3d_run(g1, sph, u0, steps, 0)
        else:
            ref_o, _ = po.adi3d_run(g0, po.MaterialSpec(), u0, 3, 0, True)
            ex_o, _ = po.adi3d_run(g1, sph, u0, steps, 0, True)
        assert _rel(gs.reference, ref_o) <= TOL
        assert _rel(gs.exit_field, ex_o) <= TOL
        want = off.farfield_3d(gs.exit_field, 1024, -0.05, 0.05, K, dx, dx,
                               reference=gs.reference, export_rows=64, export_cols=64)
        assert ff.shape == want.shape == (64, 64)
        assert _rel(ff, want) <= TOL
        # the saved datasets: projections resized to the export dimensions on the device
        written = gs.save(str(tmp_path))
        names = sorted(os.path.basename(w) for w in written)
        assert names == ["exitField.npy", "exitIntensity.npy", "exitPhase.npy", "farField.npy"]
        d = os.path.join(str(tmp_path), "data")
        assert _rel(np.load(os.path.join(d, "farField.npy")), want) <= TOL
        ei = np.load(os.path.join(d, "exitIntensity.npy"))
        want_ei = off.resize_matrix(np.abs(gs.exit_field) ** 2, 64, 64)
        assert ei.shape == (64, 64) and _rel(ei, want_ei) <= 1e-13
        ef = np.load(os.path.join(d, "exitField.npy"))
        assert _rel(ef, off.resize_matrix(gs.exit_field.real, 64, 64)) <= 1e-13


def test_resized_post_quantities_match_resize_matrix():
    """pxp_get_post_resized: the device's |u|^2, Re u and arg u of a 3-D
    field resized by resizeMatrix equal the restatement on the same field;
    export dimensions not smaller in both directions return the field."""
    from paxpro_b200 import _capi
    s, dx = _solver3d("fft3d", 256)
    with s:
        u = s.get_last_solution()
        for q, f in ((_capi.POST_ABS2, lambda a: np.abs(a) ** 2), (_capi.POST_REAL, np.real),
                     (_capi.POST_ARG, np.angle)):
            got = s.get_post_resized(q, 100, 60)
            want = off.resize_matrix(f(u), 100, 60)
            assert got.shape == (100, 60)
            np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-15)
        full = s.get_post_resized(_capi.POST_ABS2, 300, 60)
        np.testing.assert_allclose(full, np.abs(u) ** 2, rtol=4e-16 * 4, atol=0)
