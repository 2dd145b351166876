"""Steps replayed from a captured CUDA graph give the same fields, bit for
bit, as the same steps launched one by one (PXP_STEP_GRAPHS=0).  The switch
is read once per process, so each mode runs in its own interpreter."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, {root!r})
import paxpro_b200 as pxp
from paxpro_b200 import workloads as wl
kind, n, nsteps, out = sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), sys.argv[4]
xmin, xmax = -500.0, 500.0
dx = wl.step_for_nodes(xmin, xmax, n)
dz = 1000.0
spec = pxp.ProblemSpec(kind=pxp.ADI if kind == "adi" else pxp.FFT_SOLVER_3D,
                       x=pxp.Disc(xmin, xmax, dx), y=pxp.Disc(xmin, xmax, dx),
                       z=pxp.Disc(0.0, nsteps * dz, dz), wavenumber=wl.K, save_every=25)
# one sphere crossed mid-run: the run splits into graph blocks, direct steps
# at the sphere, and more graph blocks
sph = [pxp.Sphere(20.0, -30.0, 61.0 * dz, 150.0, 4e-5, 2e-6)]
x = xmin + dx * np.arange(n)
u0 = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / 200.0 ** 2).astype(np.complex128)
with pxp.Solver(spec) as s:
    s.set_material_spheres(sph)
    s.set_initial_conditions(np.asfortranarray(u0))
    s.step(nsteps // 2)
    s.step(nsteps - nsteps // 2)
    res = [s.get_last_solution()] + [s.get_saved(i) for i in range(s.num_saved())]
np.save(out, np.stack(res))
"""


def _run(kind, n, nsteps, graphs, tmp_path):
    out = str(tmp_path / f"{kind}_{n}_{graphs}.npy")
    # the FFT3D launch variant is pinned: each process would otherwise time
    # the variants itself, and radix 8 and radix 16 round differently
    env = dict(os.environ, PXP_STEP_GRAPHS="1" if graphs else "0", PXP_FFT3D_VARIANT="1")
    subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT), kind, str(n), str(nsteps), out],
                   check=True, env=env, timeout=600)
    return np.load(out)


@pytest.mark.parametrize("kind,n", [("adi", 256), ("adi", 1024), ("fft3d", 256), ("fft3d", 1024)])
def test_graph_replay_matches_direct_launches(kind, n, tmp_path):
    a = _run(kind, n, 150, True, tmp_path)
    b = _run(kind, n, 150, False, tmp_path)
    assert a.shape == b.shape and a.shape[0] == 1 + 150 // 25
    assert np.array_equal(a, b)
    assert np.all(np.isfinite(a))
