"""The oracle against the reference's own propagation code.

oracle/_ref/libpaxpro_refpin.so is the reference's solver, simulation,
source and geometry sources (src/crancNicholson.cpp,
src/alternatingDirectionSolver.cpp, src/fftSolver2D.cpp, src/fftSolver3D.cpp,
src/solver*.cpp, src/paraxialSimulation.cpp, ...) compiled where they lie,
against stand-ins for the absent third-party headers (oracle/refshim/:
Armadillo containers, FFTW3's interface over the oracle's FFT, HDF5/jsoncpp/
VISA declarations).  Each case drives the reference classes as a user
program does (setSolver, setInitialConditions, Solver::step) and requires
the oracle's restatement to give the same bits at every saved step.  The
FFT is the one shared piece (FFTW itself is absent), so these cases pin
everything around it: the propagator and transmission factors, the CN and
ADI matrices, their Thomas solves and boundary terms, the refraction
integral, the absorber, the sources and the saved-slice averages.

The GPU parity tests compare the CUDA path with the oracle, so through these
cases they compare it with the reference's own code."""
import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.skipif(po.refpin() is None,
                                reason="reference pin library not built (no reference tree)")


def _same_bits(a, b):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def _waveguide(n, kind, nsteps, dz, waist=15.0, xmin=-250.0, xmax=250.0):
    p = wl.Problem2D("pin", kind, xmin, xmax, wl.step_for_nodes(xmin, xmax, n), 0.0,
                     (nsteps + 1) * dz, dz, nsteps, waist, wl.Waveguide())
    d, b = p.material()
    g = po.grid(p.xmin, p.xmax, p.dx, p.zmin, p.zmax, p.dz, wl.K)
    return g, po.MaterialSpec(po.MAT_XTABLE, delta_table=d, beta_table=b), p.initial_field()


@pytest.mark.parametrize("n,nsteps", [(256, 60), (2048, 40), (300, 30), (9, 20)])
def test_fft_solver_2d_matches_reference_build(n, nsteps):
    g, spec, u0 = _waveguide(n, "fft", nsteps, 1000.0)
    o, os_ = po.fft2d_run(g, spec, u0, nsteps, 10)
    r, rs = po.ref_run2d(po.REF_FFT_SOLVER_2D, g, spec, u0, nsteps, 10)
    assert _same_bits(o, r)
    assert len(os_) == len(rs) == nsteps // 10
    assert all(_same_bits(a, b) for a, b in zip(os_, rs))


def test_fft_solver_2d_full_waveguide_workload_matches_reference_build():
    """The FFTSolver2D workload as timed: Nx = 2048, 4000 steps of 1 um,
    saves every 100 steps."""
    p = wl.waveguide_fft2d()
    d, b = p.material()
    g = po.grid(p.xmin, p.xmax, p.dx, p.zmin, p.zmax, p.dz, wl.K)
    spec = po.MaterialSpec(po.MAT_XTABLE, delta_table=d, beta_table=b)
    o, os_ = po.fft2d_run(g, spec, p.initial_field(), p.nsteps, 100)
    r, rs = po.ref_run2d(po.REF_FFT_SOLVER_2D, g, spec, p.initial_field(), p.nsteps, 100)
    assert len(os_) == 40
    assert all(_same_bits(a, b) for a, b in zip(os_, rs))
    assert _same_bits(o, r)


@pytest.mark.parametrize("n,nsteps,transparent", [(512, 80, False), (300, 40, False),
                                                  (17, 30, False), (256, 60, True),
                                                  (100, 30, True)])
def test_crank_nicholson_matches_reference_build(n, nsteps, transparent):
    g, spec, u0 = _waveguide(n, "cn", nsteps, 500.0, waist=40.0 if transparent else 15.0)
    o, os_ = po.cn2d_run(g, spec, u0, nsteps, 10, transparent=transparent)
    r, rs = po.ref_run2d(po.REF_CRANK_NICHOLSON, g, spec, u0, nsteps, 10, transparent=transparent)
    assert all(_same_bits(a, b) for a, b in zip(os_, rs))
    assert _same_bits(o, r)


def test_crank_nicholson_at_the_timed_size_matches_reference_build():
    """CrankNicholson at the timed workload's grid (Nx = 4096, dz = 0.5 um),
    the first 800 of its 8000 steps."""
    p = wl.waveguide_cn()
    nsteps = 800
    d, b = p.material()
    g = po.grid(p.xmin, p.xmax, p.dx, p.zmin, (nsteps + 1) * p.dz, p.dz, wl.K)
    spec = po.MaterialSpec(po.MAT_XTABLE, delta_table=d, beta_table=b)
    o, os_ = po.cn2d_run(g, spec, p.initial_field(), nsteps, 100)
    r, rs = po.ref_run2d(po.REF_CRANK_NICHOLSON, g, spec, p.initial_field(), nsteps, 100)
    assert all(_same_bits(a, b) for a, b in zip(os_, rs))
    assert _same_bits(o, r)


def _adi_case(n, nsteps, spheres, half_width=500.0):
    dx = wl.step_for_nodes(-half_width, half_width, n)
    g = po.grid(-half_width, half_width, dx, 0.0, (nsteps + 1) * 1000.0, 1000.0, wl.K)
    return g, po.MaterialSpec(po.MAT_SPHERES, spheres=spheres)


@pytest.mark.parametrize("n,tbc", [(64, False), (64, True), (50, False), (33, True)])
def test_adi_matches_reference_build(n, tbc):
    """ADI across a sphere (both half-step planes meet it), Dirichlet and
    transparent ends, sizes that are and are not powers of two."""
    nsteps = 5
    g, spec = _adi_case(n, nsteps, [(30.0, -20.0, 2500.0, 350.0, 4.5e-5, 3.6e-6),
                                    (-200.0, 150.0, 3000.0, 120.0, 2e-5, 1e-6)])
    rng = np.random.default_rng(n)
    u0 = np.asfortranarray(np.ones((n, n)) + 0.05 * rng.standard_normal((n, n)) + 0j)
    o, os_ = po.adi3d_run(g, spec, u0, nsteps, 1, use_tbc=tbc)
    r, rs = po.ref_run3d(po.REF_ADI, g, spec, u0, nsteps, 1, use_tbc=tbc)
    assert all(_same_bits(a, b) for a, b in zip(os_, rs))
    assert _same_bits(o, r)


@pytest.mark.parametrize("n,absorber", [(64, (0.0, 0.0)), (64, (100.0, 50.0)),
                                        (128, (0.0, 0.0)), (33, (0.0, 0.0)), (50, (80.0, 40.0))])
def test_fft_solver_3d_matches_reference_build(n, absorber):
    """FFTSolver3D through sphere rims, where the refraction integral between
    the step's planes runs (src/fftSolver3D.cpp:122-156, 253-273), with and
    without the absorbing boundary."""
    nsteps = 6
    dx = wl.step_for_nodes(-1000.0, 1000.0, n)
    g = po.grid(-1000.0, 1000.0, dx, 0.0, (nsteps + 1) * 1000.0, 1000.0, wl.K)
    spec = po.MaterialSpec(po.MAT_SPHERES, spheres=[(0.0, 0.0, 2500.0, 900.0, 4.5e-5, 3.6e-6),
                                                    (400.0, -300.0, 4200.0, 300.0, 1e-5, 2e-7)])
    u0 = np.ones((n, n), dtype=np.complex128, order="F")
    o, os_ = po.fft3d_run(g, spec, u0, nsteps, 2, *absorber)
    r, rs = po.ref_run3d(po.REF_FFT_SOLVER_3D, g, spec, u0, nsteps, 2, False, *absorber,
                         threads=4)
    assert all(_same_bits(a, b) for a, b in zip(os_, rs))
    assert _same_bits(o, r)


@pytest.mark.parametrize("ratio", [2, 3, 4])
def test_saved_block_averages_match_reference_build(ratio):
    """Solver3D::copyCurrentSolution's downsampled slices (src/solver3D.cpp:
    94-112) against the oracle's block average of the same fields."""
    n, nsteps = 64, 4
    g, spec = _adi_case(n, nsteps, [(0.0, 0.0, 2000.0, 300.0, 4.5e-5, 3.6e-6)])
    rng = np.random.default_rng(ratio)
    u0 = np.asfortranarray(np.ones((n, n)) + 0.1 * rng.standard_normal((n, n)) + 0j)
    cube = po.ref_saved_cube(po.REF_ADI, g, spec, u0, nsteps, ratio, 1)
    _, fields = po.adi3d_run(g, spec, u0, nsteps, 1)
    assert _same_bits(cube[0], po.block_average(u0, ratio))
    for step in range(1, nsteps + 1):
        assert _same_bits(cube[step], po.block_average(fields[step - 1], ratio))


@pytest.mark.parametrize("dim", [2, 3])
def test_gaussian_beam_source_matches_reference_build(dim):
    n = 257
    dx = wl.step_for_nodes(-400.0, 400.0, n)
    g = po.grid(-400.0, 400.0, dx, 0.0, 2000.0, 1000.0, wl.K)
    r = po.ref_source_field(dim, g, 0, 0.1569, waist=35.0, cx=12.0, cy=-7.0, amplitude=1.5)
    if dim == 2:
        o = po.gaussian_beam_2d(g, 0.1569, 35.0, center=12.0, amplitude=1.5)
    else:
        o = po.gaussian_beam_3d(g, 0.1569, 35.0, cx=12.0, cy=-7.0, amplitude=1.5)
    assert _same_bits(o, r)


def test_plane_wave_source_matches_reference_build():
    n = 64
    dx = wl.step_for_nodes(-500.0, 500.0, n)
    g = po.grid(-500.0, 500.0, dx, 0.0, 2000.0, 1000.0, wl.K)
    r = po.ref_source_field(3, g, 1, 0.1, amplitude=1.0)
    assert np.array_equal(r, np.ones((n, n), dtype=np.complex128))


def test_node_count_matches_reference_build():
    from paxpro_b200 import _capi
    lib = _capi.lib()
    cases = [(-250.0, 250.0, 500.0 / 2047), (-250.0, 250.0, 500.0 / 2048), (0.0, 4e6, 1000.0),
             (-1000.0, 1000.0, 2000.0 / 4095), (-500.0, 500.0, 1000.0 / 1023), (-1.0, 1.0, 0.3)]
    for mn, mx, st in cases:
        want = po.refpin().ref_node_count(mn, mx, st)
        assert po.node_count(mn, mx, st) == want
        assert lib.pxp_node_count(mn, mx, st) == want


def test_csg_material_matches_reference_geometry_classes():
    """CSGMaterial::getXrayMatProp of a scene built from the reference's own
    geom:: classes (src/shape.cpp, src/geometry.cpp, src/materialFunction.cpp)
    against the oracle's evaluation of the flattened scene (the form the
    device takes, pxp_set_material_csg) and the Python classes, at random
    points around every object: equal values at every point."""
    import ctypes as C

    from paxpro_b200 import csg

    from csg_geometry import geometry, reference_arrays

    mods = geometry()
    spec = po.MaterialSpec(po.MAT_CSG, csg=csg.flatten(mods))
    g = po.grid(-500.0, 500.0, 1.0, 0.0, 8000.0, 1000.0, 62.83)
    rng = np.random.default_rng(11)
    centres = np.array([(0.0, 0.0, 3000.0), (100.0, -100.0, 4000.0), (-150.0, 50.0, 5000.0),
                        (-300.0, 300.0, 6000.0), (20.0, 0.0, 3000.0)])
    npts = 6000
    xyz = centres[np.arange(npts) % len(centres)] + rng.uniform(-200.0, 200.0, (npts, 3))
    xyz = np.ascontiguousarray(xyz)
    out = np.zeros(2 * npts)
    m, p, s, o = reference_arrays()
    rp = po.refpin()
    rc = rp.ref_csg_eval(m, len(m), p, s, o, xyz.ctypes.data_as(C.POINTER(C.c_double)), npts,
                         out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    hits = 0
    for i in range(npts):
        x, y, z = xyz[i]
        want = (out[2 * i], out[2 * i + 1])
        assert po.material_eval(spec, g, x, y, z) == want, (x, y, z)
        assert csg.material(mods, x, y, z) == want, (x, y, z)
        hits += want[0] != 0.0
    assert 300 < hits < npts - 300  # inside and outside points of several parts
