"""Per-step flux sums fused into the 2-D step kernels (post::Transmittivity's
trapezoid integral, src/transmittivity.cpp:30-41) against the same sums
taken on the host from the saved fields: the same terms (pow(abs(u), 2),
weights 1 at the window's ends and 2 between), summed exactly with
math.fsum; the device's compensated sums agree to a few ulps."""
import math

import numpy as np
import pytest

from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def trapezoid_sum(u, a, b):
    """trapezoidalIntegrateIntensityZ without dx/2, correctly rounded."""
    terms = [abs(u[a]) ** 2, abs(u[b]) ** 2] + [2.0 * abs(u[i]) ** 2 for i in range(a + 1, b)]
    return math.fsum(terms)


def _run(kind, n, precision, steps, planes, transparent=False):
    import paxpro_b200 as pxp
    L = 500.0
    dx = wl.step_for_nodes(-L / 2, L / 2, n)
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D if kind == "fft" else pxp.CRANK_NICHOLSON,
                           x=pxp.Disc(-L / 2, L / 2, dx), z=pxp.Disc(0.0, steps * 500.0, 500.0),
                           wavenumber=wl.K, precision=precision, save_every=1,
                           transparent_bc=transparent)
    s = pxp.Solver(spec)
    x = -L / 2 + dx * np.arange(n)
    if planes:
        per = 2 if kind == "cn" else 1
        zs = 500.0 * np.arange(1, steps + 1)
        d = np.stack([np.where(np.abs(x - 1e-4 * z * z / 500.0) < 25.0, 0.0, 7.5e-6)
                      for z in zs for _ in range(per)])
        s.set_material_planes(d, np.full_like(d, 1e-8), 1, steps)
    else:
        s.set_material_table(np.where(np.abs(x) < 25.0, 0.0, 7.5e-6), np.full(n, 1e-8))
    s.set_initial_conditions(np.exp(-(x - 5.0) ** 2 / 15.0 ** 2).astype(np.complex128))
    rng = np.random.default_rng(n + steps)
    a = rng.integers(0, n // 2, steps)
    b = a + rng.integers(0, n // 2, steps)
    a[0], b[0] = 0, n - 1                 # whole line
    a[1], b[1] = 7, 7                     # single point: 2 |u|^2
    s.set_flux_windows(1, a, b)
    return s, a, b


@pytest.mark.parametrize("kind,n,precision,planes", [
    ("fft", 1024, 0, False), ("fft", 256, 1, True), ("fft", 8192, 0, False),
    ("fft", 16384, 0, False),
    ("cn", 1024, 0, False), ("cn", 512, 0, True), ("cn", 16, 0, False), ("cn", 4096, 1, False)])
def test_fused_flux_matches_saved_fields(kind, n, precision, planes):
    steps = 24
    s, a, b = _run(kind, n, precision, steps, planes)
    with s:
        s.step(10)
        part = s.get_flux(1, steps)
        assert np.all(np.isfinite(part[:10])) and np.all(np.isnan(part[10:]))
        s.step(steps - 10)
        got = s.get_flux(1, steps)
        saved = [s.get_saved(k) for k in range(s.num_saved())]
        want = np.array([trapezoid_sum(saved[k], a[k], b[k]) for k in range(steps)])
        assert want.max() > 0
        np.testing.assert_allclose(got, want, rtol=1e-14, atol=0)
        last = s.get_last_solution()
        assert s.field_flux(3, n - 5) == pytest.approx(trapezoid_sum(last, 3, n - 5), rel=1e-14)


def test_flux_windows_validation_and_clear():
    import paxpro_b200 as pxp
    s, a, b = _run("fft", 256, 0, 6, False)
    with s:
        with pytest.raises(pxp.PxpError):
            s.set_flux_windows(1, [5], [4])
        with pytest.raises(pxp.PxpError):
            s.set_flux_windows(1, [0], [256])
        s.set_flux_windows(1, [], [])
        s.step(6)
        with pytest.raises(pxp.PxpError):
            s.get_flux(1, 1)
