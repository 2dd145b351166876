"""Sampled material planes for the 3-D solvers (any MaterialFunction the
host evaluates): pxp_set_material_planes with the planes the reference
samples -- FFTSolver3D: per step the (delta, beta) its refraction applies,
refraction integral included (src/fftSolver3D.cpp:122-156, 253-273); ADI:
the x and y half-step planes (src/alternatingDirectionSolver.cpp:21, 91) --
gives the oracle's fields for the material the planes were sampled from
(FP64, <= 1e-10 relative L2 at every saved step).  A z-invariant medium
goes through pxp_set_material_table as one plane."""
import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu
TOL = 1e-10

SPHERES = [(30.0, -20.0, 2500.0, 350.0, 4.5e-5, 3.6e-6),
           (-200.0, 150.0, 3000.0, 120.0, 2e-5, 1e-6)]


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _case(kind, n, nsteps, tbc=False, spec=None):
    import paxpro_b200 as pxp
    dx = wl.step_for_nodes(-500.0, 500.0, n)
    g = po.grid(-500.0, 500.0, dx, 0.0, nsteps * 1000.0, 1000.0, wl.K)
    spec = spec or po.MaterialSpec(po.MAT_SPHERES, spheres=SPHERES)
    rng = np.random.default_rng(n)
    u0 = np.asfortranarray(np.ones((n, n)) + 0.05 * rng.standard_normal((n, n)) + 0j)
    k = pxp.ADI if kind == 4 else pxp.FFT_SOLVER_3D
    ps = pxp.ProblemSpec(kind=k, x=pxp.Disc(-500.0, 500.0, dx), y=pxp.Disc(-500.0, 500.0, dx),
                         z=pxp.Disc(0.0, nsteps * 1000.0, 1000.0), wavenumber=wl.K,
                         transparent_bc=tbc, save_every=1)
    run = po.adi3d_run if kind == 4 else po.fft3d_run
    ref_out, ref_saves = (po.adi3d_run(g, spec, u0, nsteps, 1, tbc) if kind == 4
                          else po.fft3d_run(g, spec, u0, nsteps, 1))
    return pxp, ps, g, spec, u0, ref_out, ref_saves


@pytest.mark.parametrize("kind,n,tbc", [(4, 64, False), (4, 100, True), (3, 128, False),
                                        (3, 64, False)])
def test_sampled_planes_match_the_oracle(kind, n, tbc):
    nsteps = 5
    pxp, ps, g, spec, u0, ref_out, ref_saves = _case(kind, n, nsteps, tbc)
    d, b = po.material_planes(g, spec, kind, 1, nsteps)
    with pxp.Solver(ps) as s:
        s.set_material_planes(d, b, 1, nsteps)
        s.set_initial_conditions(u0)
        s.step(2)            # planes in two calls: the chunk boundary
        s.step(nsteps - 2)
        saves = [s.get_saved(i) for i in range(s.num_saved())]
    assert len(saves) == nsteps
    errs = [_rel(a, r) for a, r in zip(saves, ref_saves)]
    assert max(errs) <= TOL, errs
    assert np.std(np.abs(saves[-1])) > 1e-3


def test_planes_in_blocks_and_outside_their_range():
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi
    nsteps = 6
    pxp, ps, g, spec, u0, ref_out, ref_saves = _case(4, 64, nsteps)
    with pxp.Solver(ps) as s:
        s.set_initial_conditions(u0)
        for first in (1, 4):  # two blocks of three steps, as the C++ API feeds them
            d, b = po.material_planes(g, spec, 4, first, 3)
            s.set_material_planes(d, b, first, 3)
            s.step(3)
        out = s.get_last_solution()
        # step 7 has no plane
        assert _capi.lib().pxp_step(s._h, 1) == _capi.PXP_ERR_INVALID
    assert _rel(out, ref_out) <= TOL


@pytest.mark.parametrize("kind", [3, 4])
def test_z_invariant_table_for_3d_kinds(kind):
    """A medium that does not change along z (a cylinder along z longer than
    the run): one table for every step."""
    from paxpro_b200 import csg
    col = csg.Module()
    col.add(csg.Part(delta=2e-5, beta=3e-7).add(csg.Cylinder(150.0, 1e7)))
    spec = po.MaterialSpec(po.MAT_CSG, csg=csg.flatten([col]))
    nsteps = 4
    pxp, ps, g, spec, u0, ref_out, ref_saves = _case(kind, 64, nsteps, spec=spec)
    d, b = po.material_planes(g, spec, kind, 1, 1)
    with pxp.Solver(ps) as s:
        s.set_material_table(d[0], b[0])
        s.set_initial_conditions(u0)
        s.step(nsteps)
        out = s.get_last_solution()
    assert _rel(out, ref_out) <= TOL
    assert np.std(np.abs(out)) > 1e-4
