"""FFTSolver3D and ADI with a constructive-solid-geometry material evaluated
on the device, against the oracle with the same geometry: FP64 <= 1e-10
relative L2 at every saved step."""
import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import csg
from paxpro_b200 import workloads as wl

from csg_geometry import geometry

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("kind", ["fft3d", "adi"])
def test_csg_material_parity(kind):
    import paxpro_b200 as pxp
    po.set_fft_parallel(True)
    n, dz, nsteps = 256, 1000.0, 7
    xmin, xmax = -500.0, 500.0
    dx = wl.step_for_nodes(xmin, xmax, n)
    mods = geometry()
    g = po.grid(xmin, xmax, dx, 0.0, nsteps * dz, dz, wl.K)
    spec_o = po.MaterialSpec(po.MAT_CSG, csg=csg.flatten(mods))
    u0 = np.ones((n, n), dtype=np.complex128, order="F")
    run = po.fft3d_run if kind == "fft3d" else po.adi3d_run
    ref_out, ref_saves = run(g, spec_o, u0, nsteps, 1)
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_3D if kind == "fft3d" else pxp.ADI,
                           x=pxp.Disc(xmin, xmax, dx), y=pxp.Disc(xmin, xmax, dx),
                           z=pxp.Disc(0.0, nsteps * dz, dz), wavenumber=wl.K, save_every=1)
    with pxp.Solver(spec) as s:
        s.set_material_csg(mods)
        s.set_initial_conditions(u0)
        s.step(nsteps)
        saves = [s.get_saved(i) for i in range(s.num_saved())]
        out = s.get_last_solution()
    assert len(saves) == len(ref_saves) == nsteps
    errs = [_rel(a, b) for a, b in zip(saves, ref_saves)]
    assert max(errs) <= 1e-10, errs
    assert _rel(out, ref_out) <= 1e-10
    assert np.std(np.abs(out)) > 1e-4   # the geometry left a mark
