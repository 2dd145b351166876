"""The pipelined one-wave ADI vacuum kernel (staging in per-group stages,
each system group solving as soon as its rows land; PXP_ADI_PIPE=1)
against the unpipelined one (PXP_ADI_PIPE=0, each run in a child
process because the switch is read once per process): the two share the
solve's arithmetic, so their fields are equal bit for bit, for both half
steps (x: systems adjacent in memory; y: systems as rows), with saves, at
every system length the one-wave kernel solves and on grids it pads."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import paxpro_b200 as pxp
from paxpro_b200 import workloads as wl
n = int(sys.argv[2])
dx = wl.step_for_nodes(-500.0, 500.0, n)
spec = pxp.ProblemSpec(kind=pxp.ADI, x=pxp.Disc(-500.0, 500.0, dx), y=pxp.Disc(-500.0, 500.0, dx),
                       z=pxp.Disc(0.0, 4e4, 1000.0), wavenumber=wl.K, save_every=7)
rng = np.random.default_rng(n)
u0 = np.asfortranarray(np.ones((n, n)) + 0.05 * rng.standard_normal((n, n)) + 0j)
with pxp.Solver(spec) as s:
    s.set_material_spheres([pxp.Sphere(20.0, -10.0, 9000.0, 150.0, 4.5e-5, 3.6e-6)])
    s.set_initial_conditions(u0)
    s.step(30)
    out = [s.get_last_solution()] + [s.get_saved(i) for i in range(s.num_saved())]
np.save(sys.argv[3], np.stack(out))
"""


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 33, 300, 513, 1000])
def test_pipelined_wave_kernel_equals_unpipelined(n, tmp_path):
    res = {}
    for pipe in ("1", "0"):
        path = str(tmp_path / f"adi_{n}_{pipe}.npy")
        env = dict(os.environ, PXP_ADI_PIPE=pipe)
        r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT, str(n), path], env=env,
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        res[pipe] = np.load(path)
    assert res["1"].shape[0] == 1 + 30 // 7
    assert np.array_equal(res["1"].view(np.uint64), res["0"].view(np.uint64))
    assert np.std(np.abs(res["1"][0])) > 1e-3  # the sphere was crossed
