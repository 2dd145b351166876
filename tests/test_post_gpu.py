"""Post-processing modules (device-side reductions) and the save path: the
device's |u|, arg u, Re u, |u|^2 and max |u| against numpy on the same
fields read back, module shapes and names as the reference's post:: modules,
and the exported datasets and group attributes."""
import json
import os

import numpy as np
import pytest

from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _fft3d(ratio=1, precision=0):
    import paxpro_b200 as pxp
    n, dz, nsteps = 256, 1000.0, 6
    xmin, xmax = -500.0, 500.0
    dx = wl.step_for_nodes(xmin, xmax, n)
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_3D, x=pxp.Disc(xmin, xmax, dx, ratio),
                           y=pxp.Disc(xmin, xmax, dx, ratio), z=pxp.Disc(0.0, nsteps * dz, dz),
                           wavenumber=wl.K, precision=precision, save_every=2)
    s = pxp.Solver(spec, keep_initial=True)
    s.set_material_spheres([pxp.Sphere(10.0, -20.0, 2000.0, 150.0, 4e-5, 2e-6)])
    x = xmin + dx * np.arange(n)
    u0 = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / 150.0 ** 2 + 0.3j * x[None, :] / 50.0)
    s.set_initial_conditions(np.asfortranarray(u0.astype(np.complex128)))
    s.step(nsteps)
    return s, u0


def test_device_reductions_match_numpy_on_the_same_fields():
    from paxpro_b200 import _capi
    s, _ = _fft3d()
    with s:
        last = s.get_last_solution()
        np.testing.assert_allclose(s.get_post(_capi.POST_ABS), np.abs(last), rtol=1e-15, atol=0)
        np.testing.assert_allclose(s.get_post(_capi.POST_ABS2), np.abs(last) ** 2, rtol=4e-16 * 4, atol=0)
        np.testing.assert_array_equal(s.get_post(_capi.POST_REAL), last.real)
        np.testing.assert_allclose(s.get_post(_capi.POST_ARG), np.angle(last), rtol=0, atol=2e-15)
        saved = [s.get_saved(k) for k in range(s.num_saved())]
        for k, f in enumerate(saved):
            np.testing.assert_allclose(s.get_post(_capi.POST_ABS, k), np.abs(f), rtol=1e-15, atol=0)
        assert s.saved_max_abs() == pytest.approx(max(np.abs(f).max() for f in saved), rel=1e-15)


def test_modules_shapes_values_and_export(tmp_path):
    from paxpro_b200 import post
    s, u0 = _fft3d(ratio=2)
    with s:
        amp = post.Intensity().result(s)
        assert amp.shape == (128, 128, 1 + s.num_saved())
        np.testing.assert_allclose(amp[:, :, 0], np.abs(post._block_average(u0, 128)), rtol=1e-14)
        np.testing.assert_allclose(amp[:, :, 1], np.abs(s.get_saved(0)), rtol=1e-15)
        u8 = post.IntensityUint8().result(s)
        assert u8.dtype == np.uint8 and u8.max() == 255
        lg = post.LogIntensityUint8().result(s)
        assert lg.dtype == np.uint8 and lg.max() == 255
        ph = post.Phase().result(s)
        assert ph.shape == amp.shape and np.all(np.abs(ph) <= np.pi)
        ex = post.ExitIntensity().result(s)
        assert ex.shape == (256, 256)
        np.testing.assert_allclose(ex, np.abs(s.get_last_solution()) ** 2, rtol=2e-15)
        files = post.save(s, str(tmp_path / "run"), [post.Intensity(), post.Phase(),
                                                      post.ExitField(), post.ExitPhase()],
                          description="sphere test")
        names = sorted(os.path.basename(f) for f in files)
        assert names == ["amplitude.npy", "exitField.npy", "exitPhase.npy", "phase.npy"]
        back = np.load(tmp_path / "run" / "data" / "amplitude.npy")
        assert back.flags.f_contiguous and np.array_equal(back, amp)
        attrs = json.load(open(tmp_path / "run" / "data" / "attributes.json"))
        assert attrs["solver"] == "FFTSolver3D" and attrs["description"] == "sphere test"
        assert attrs["wavenumber"] == pytest.approx(wl.K) and attrs["dz"] == 1000.0


def test_2d_solver_field_quantity_is_points_by_slices():
    import paxpro_b200 as pxp
    from paxpro_b200 import post
    p = wl.waveguide_fft2d(nsteps=5)
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D, x=pxp.Disc(p.xmin, p.xmax, p.dx),
                           z=pxp.Disc(p.zmin, 5 * p.dz, p.dz), wavenumber=wl.K, save_every=1)
    with pxp.Solver(spec, keep_initial=True) as s:
        d, b = p.material()
        s.set_material_table(d, b)
        s.set_initial_conditions(p.initial_field())
        s.step(5)
        amp = post.Intensity().result(s)
        assert amp.shape == (2048, 6)  # the initial condition and every step
        np.testing.assert_allclose(amp[:, -1], np.abs(s.get_last_solution()), rtol=1e-15)
        assert post.ExitField().result(s).shape == (2048,)
