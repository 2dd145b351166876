"""GPU parity of ADI (2 transverse dims) against the CPU oracle, through the
C ABI.  FP64: <= 1e-10 relative L2 at every saved step; FP32 served mode:
<= 1e-4 relative L2 of the intensity.

The oracle's ADI is serial over n*n unknowns per half step (as the
reference's), so the full-size case (config 1: 1024^2, sphere R = 200 nm at
z = 1 mm) is checked over the steps around the sphere crossing by starting
the grid five steps before the sphere plane."""
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


def _run_both(n, zmin, nsteps, dz, spheres, u0=None, use_tbc=False, precision=0, save_every=1,
              L=1000.0, chunks=1):
    import paxpro_b200 as pxp
    xmin, xmax = -L / 2, L / 2
    dx = wl.step_for_nodes(xmin, xmax, n)
    zmax = zmin + nsteps * dz
    if u0 is None:
        u0 = np.ones((n, n), dtype=np.complex128, order="F")
    g = po.grid(xmin, xmax, dx, zmin, zmax, dz, wl.K)
    ref_out, ref_saves = po.adi3d_run(g, po.MaterialSpec(po.MAT_SPHERES, spheres=spheres), u0,
                                      nsteps, save_every, use_tbc)
    spec = pxp.ProblemSpec(kind=pxp.ADI, x=pxp.Disc(xmin, xmax, dx), y=pxp.Disc(xmin, xmax, dx),
                           z=pxp.Disc(zmin, zmax, dz), wavenumber=wl.K, precision=precision,
                           transparent_bc=use_tbc, save_every=save_every)
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


def test_sphere_adi_fp64_sphere_crossing_full_size():
    p = wl.sphere_adi()
    sph = p.spheres
    out, saves, ref_out, ref_saves = _run_both(1024, 1.0e6 - 5 * p.dz, 10, p.dz, sph)
    assert len(saves) == len(ref_saves) == 10
    errs = [_rel(a, b) for a, b in zip(saves, ref_saves)]
    assert max(errs) <= FP64_TOL, errs
    # the sphere leaves a mark: the field is not a plane wave any more
    assert np.std(np.abs(out)) > 1e-3


@pytest.mark.parametrize("n", [64, 256, 512, 2048])
def test_adi_fp64_sizes(n):
    sph = [(30.0, -40.0, 3000.0, 150.0, 4.5e-5, 3.6e-6), (-100.0, 80.0, 5200.0, 90.0, 2e-5, 1e-6)]
    nsteps = 8 if n == 2048 else 12
    out, saves, ref_out, ref_saves = _run_both(n, 0.0, nsteps, 500.0, sph, chunks=2)
    assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL


def test_adi_fp64_many_steps_small_grid():
    sph = [(0.0, 0.0, 20000.0, 200.0, 4.5e-5, 3.6e-6)]
    out, saves, ref_out, ref_saves = _run_both(128, 0.0, 200, 1000.0, sph, save_every=20)
    assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL


def test_adi_transparent_boundary():
    n = 128
    L = 1000.0
    dx = wl.step_for_nodes(-L / 2, L / 2, n)
    g = po.grid(-L / 2, L / 2, dx, 0.0, 1e5, 1000.0, wl.K)
    u0 = po.gaussian_beam_3d(g, wl.WAVELENGTH, 150.0, cx=60.0, cy=-40.0)
    sph = [(0.0, 0.0, 4000.0, 120.0, 3e-5, 1e-6)]
    out, saves, ref_out, ref_saves = _run_both(n, 0.0, 40, 1000.0, sph, u0=u0, use_tbc=True,
                                               save_every=10)
    assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL


def test_adi_fp32_served_intensity():
    sph = [(0.0, 0.0, 20000.0, 200.0, 4.5e-5, 3.6e-6)]
    out, saves, ref_out, ref_saves = _run_both(256, 0.0, 200, 1000.0, sph, precision=1,
                                               save_every=50)
    assert max(_int_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP32_INT_TOL


@pytest.mark.parametrize("n,use_tbc,precision", [(100, False, 0), (300, False, 0), (129, True, 0),
                                                 (200, False, 1), (5, False, 0), (33, False, 0),
                                                 (513, False, 0), (700, False, 0), (1000, False, 0),
                                                 (1500, False, 0)])
def test_adi_any_grid_size(n, use_tbc, precision):
    """ADI on grids whose size is not a power of two: every save against the
    oracle, with a sphere crossing the planes, Dirichlet and transparent
    ends.  The sphere planes run the general kernel (systems padded with
    decoupled rows to adi_padded_n), the vacuum planes the FP64 one-wave
    kernel (padded to 64 .. 1024 rows: 5 and 33 -> 64, 100 -> 128, 300 and
    513 -> 512 and 768, 700 -> 768, 1000 -> 1024) up to 1024 nodes, the
    general kernel above (1500) and in FP32 or with transparent ends."""
    sph = [(30.0, -20.0, 3000.0, 250.0, 4.5e-5, 3.6e-6)]
    x = -500.0 + wl.step_for_nodes(-500.0, 500.0, n) * np.arange(n)
    u0 = np.asfortranarray(np.exp(-(x[None, :] ** 2 + x[:, None] ** 2) / 300.0 ** 2)
                           .astype(np.complex128))
    out, saves, ref_out, ref_saves = _run_both(n, 0.0, 8, 1000.0, sph, u0=u0, use_tbc=use_tbc,
                                               precision=precision)
    assert len(saves) == len(ref_saves) == 8
    if precision == 0:
        assert max(_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP64_TOL
        assert _rel(out, ref_out) <= FP64_TOL
    else:
        assert max(_int_rel(a, b) for a, b in zip(saves, ref_saves)) <= FP32_INT_TOL
    assert np.std(np.abs(out)) > 1e-3
