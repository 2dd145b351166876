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


def test_cpp_curved_waveguide_material():
    """CurvedWaveGuideFD::getXrayMatProp of the C++ API against the
    reference's rules restated here: WaveGuideFDSimulation::getXrayMatProp
    (src/waveGuideFDSimulation.cpp:219-265: past the guide's length vacuum,
    inside with all four neighbours inside the inner material, inside at the
    border the mean of the two, outside the cladding) over
    CurvedWaveGuideFD::isInsideGuide (src/curvedWaveGuide2D.cpp:49-52), and
    the smoothed profile (:178-205)."""
    import math
    exe = build("curved2d")
    R, width, dx, dz, wgl = 40e6, 100.0, 10.0, 5000.0, 1.5e5
    clad, inner = (4.14e-5, 3.45e-6), (1e-6, 2e-8)

    def inside(x, z):
        return (2.0 * x * R + z * z > 0.0) and (2.0 * x * R + z * z < 2.0 * width * R)

    def plain(x, z):
        if z > wgl:
            return (0.0, 0.0)
        ins = inside(x, z)
        nb = inside(x + dx, z) and inside(x - dx, z) and inside(x, z + dz) and inside(x, z - dz)
        if ins and nb:
            return inner
        if ins:
            return (0.5 * (clad[0] + inner[0]), 0.5 * (clad[1] + inner[1]))
        return clad

    def smoothed(x, z):
        w = 0.1 * width
        d = 2.0 * R * x + z * z
        def logistic(a):  # 1 / (1 + exp(a)); exp overflows to inf in C++, giving 0
            return 0.0 if a > 709.78 else 1.0 / (1.0 + math.exp(a))
        f1 = logistic(-d / w)
        f2 = logistic((2 * R * width - d) / w)
        s = 1.0 - (f1 - f2)
        return (clad[0] * s, clad[1] * s)

    for sm, fn in ((0, plain), (1, smoothed)):
        out = os.path.join(OUT, f"cw_mat_{sm}.bin")
        r = subprocess.run([exe, "material", str(sm), out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = np.fromfile(out, dtype=np.float64).reshape(41, 61, 2)
        want = np.array([[fn(-400.0 + 10.0 * ix, 5000.0 * iz) for ix in range(61)]
                         for iz in range(41)])
        np.testing.assert_allclose(got, want, rtol=1e-15, atol=0)
        assert len({tuple(v) for v in want.reshape(-1, 2)}) >= (4 if sm == 0 else 3)
