"""Constructive solid geometry on the CPU: the reference's own geometry unit
tests (unittest/transformTest.cpp:4-65, known-answer K6), the reference's
CSG rules restated in Python against the oracle's C++ restatement on random
points (bit-equal: same matrices, same rounded operations), and the
construction errors of geom::Part / geom::Module."""
import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import csg

from csg_geometry import geometry


@pytest.mark.parametrize("axis,point,expect", [
    (csg.Z, (1.0, 0.0, 0.0), (0.0, -1.0, 0.0)),   # TEST(geometry, rotateZ)
    (csg.Y, (1.0, 0.0, 0.0), (0.0, 0.0, 1.0)),    # TEST(geometry, rotateY)
    (csg.X, (0.0, 1.0, 0.0), (0.0, 0.0, -1.0)),   # TEST(geometry, rotateX)
])
def test_k6_rotations(axis, point, expect):
    s = csg.Sphere(10.0).rotate(90.0, axis)
    assert np.allclose(s.transform(*point), expect, atol=1e-6)


def test_k6_translation():
    s = csg.Sphere(10.0).translate(10.0, -10.0, -3.0)   # TEST(geometry, translation)
    assert np.allclose(s.transform(1.0, -1.0, 10.0), (-9.0, 9.0, 13.0), atol=1e-6)


def test_oracle_matches_python_restatement_on_random_points():
    mods = geometry()
    spec = po.MaterialSpec(po.MAT_CSG, csg=csg.flatten(mods))
    g = po.grid(-500.0, 500.0, 1.0, 0.0, 8000.0, 1000.0, 62.83)
    rng = np.random.default_rng(7)
    hits = 0
    centres = [(0.0, 0.0, 3000.0), (100.0, -100.0, 4000.0), (-150.0, 50.0, 5000.0),
               (-300.0, 300.0, 6000.0), (20.0, 0.0, 3000.0)]
    for i in range(4000):
        c = centres[i % len(centres)]
        x, y, z = (c[k] + rng.uniform(-160.0, 160.0) for k in range(3))
        d_or, b_or = po.material_eval(spec, g, x, y, z)
        d_py, b_py = csg.material(mods, x, y, z)
        assert (d_or, b_or) == (d_py, b_py), (x, y, z)
        hits += d_py != 0.0
    assert 200 < hits < 3800   # both inside and outside points were tested


def test_construction_errors_as_the_reference():
    with pytest.raises(RuntimeError):
        csg.Part().difference(csg.Sphere(1.0))
    m = csg.Module()
    m.add(csg.Part().add(csg.Sphere(1.0)))
    with pytest.raises(RuntimeError):
        m.difference(csg.Part().add(csg.Sphere(1.0)))
