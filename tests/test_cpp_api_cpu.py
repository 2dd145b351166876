"""The C++ solver API (include/paxpro/paxpro.hpp) compiles warning-free and
links against the library; usage examples mirror the reference's
(Examples/waveguide2D.cpp pattern)."""
import os
import subprocess
import sys

import numpy as np

from tests.cpp_build import OUT, build

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from csg_geometry import geometry  # noqa: E402


def test_cpp_examples_compile_and_link():
    for name in ("waveguide2d", "sphere3d", "csg3d", "scattering3d", "curved2d"):
        assert build(name)


def test_cpp_csg_material_matches_python_geometry():
    """geom:: shapes, parts and modules of the C++ API give the material of
    the Python geometry classes at every sampled point (the device evaluates
    the flattened form of either)."""
    from paxpro_b200 import csg
    exe = build("csg3d")
    rng = np.random.default_rng(11)
    pts = np.column_stack([rng.uniform(-500.0, 500.0, 6000), rng.uniform(-500.0, 500.0, 6000),
                           rng.uniform(2700.0, 6300.0, 6000)])
    fin = os.path.join(OUT, "csg_pts.bin")
    fout = os.path.join(OUT, "csg_mat.bin")
    pts.astype(np.float64).tofile(fin)
    r = subprocess.run([exe, "material", fin, fout], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(fout, dtype=np.float64).reshape(-1, 2)
    mods = geometry()
    want = np.array([csg.material(mods, *p) for p in pts])
    assert np.array_equal(got, want)
    assert len({tuple(v) for v in want}) >= 5     # every material and vacuum were sampled
