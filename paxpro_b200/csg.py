"""Constructive solid geometry for the 3-D solvers' material hook.

Mirrors the reference's geometry classes (include/shapes.hpp,
include/geometry.hpp, src/shape.cpp, src/geometry.cpp) and its CSGMaterial
(src/materialFunction.cpp:3-13), so that a geometry built as in the
reference's examples can be handed to `Solver.set_material_csg`, which
evaluates it on the device (first module that claims a point wins; parts and
shapes scanned from the last to the first, see include/paxpro_b200.h).

A shape's `transformation` is the 4x4 matrix that maps world coordinates to
the shape's own: `translate`, `rotate` and `scale` update it exactly as
geom::Shape does (src/shape.cpp:16-58, 128-144), including the order of the
products (translate and rotate multiply on the right, scale on the left).
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

PI = math.acos(-1.0)  # as the reference writes it

SPHERE, BOX, CYLINDER = 0, 1, 2
UNION, DIFFERENCE = 0, 1
X, Y, Z = 0, 1, 2


class Shape:
    kind = -1

    def __init__(self):
        self.transformation = np.eye(4)

    def translate(self, x: float, y: float, z: float) -> "Shape":
        mat = np.eye(4)
        mat[0, 3] = -x
        mat[1, 3] = -y
        mat[2, 3] = -z
        self.transformation = self.transformation @ mat
        return self

    def rotate(self, angle_deg: float, axis: int) -> "Shape":
        angle = angle_deg * PI / 180.0
        c, s = math.cos(angle), math.sin(angle)
        mat = np.eye(4)
        if axis == X:
            mat[1, 1], mat[1, 2], mat[2, 1], mat[2, 2] = c, s, -s, c
        elif axis == Y:
            mat[0, 0], mat[0, 2], mat[2, 0], mat[2, 2] = c, -s, s, c
        else:
            mat[0, 0], mat[0, 1], mat[1, 0], mat[1, 1] = c, s, -s, c
        self.transformation = self.transformation @ mat
        return self

    def scale(self, factor: float, axis: int) -> "Shape":
        mat = np.eye(4)
        mat[axis, axis] = 1.0 / factor
        self.transformation = mat @ self.transformation
        return self

    def transform(self, x: float, y: float, z: float) -> Tuple[float, float, float]:
        """The point in the shape's coordinates, each row of the matrix summed
        left to right as the device and the oracle do."""
        T = self.transformation
        out = []
        for i in range(3):
            out.append(((T[i, 0] * x + T[i, 1] * y) + T[i, 2] * z) + T[i, 3] * 1.0)
        return tuple(out)

    def size(self) -> Tuple[float, float, float]:
        raise NotImplementedError


class Sphere(Shape):
    """geom::Sphere(radius): sqrt(x^2 + y^2 + z^2) < radius."""
    kind = SPHERE

    def __init__(self, radius: float):
        super().__init__()
        self.radius = float(radius)

    def size(self):
        return (self.radius, 0.0, 0.0)


class Box(Shape):
    """geom::Box(Lx, Ly, Lz), centred: |x| < Lx/2 and so on (strict)."""
    kind = BOX

    def __init__(self, Lx: float, Ly: float, Lz: float):
        super().__init__()
        self.L = (float(Lx), float(Ly), float(Lz))

    def size(self):
        return self.L


class Cylinder(Shape):
    """geom::Cylinder(radius, height) or (r1, r2, height): along z, centred,
    the radius growing linearly from r1 at -height/2 to r2 at +height/2."""
    kind = CYLINDER

    def __init__(self, *args: float):
        super().__init__()
        if len(args) == 2:
            self.r1 = self.r2 = float(args[0])
            self.height = float(args[1])
        elif len(args) == 3:
            self.r1, self.r2, self.height = (float(a) for a in args)
        else:
            raise TypeError("Cylinder(radius, height) or Cylinder(r1, r2, height)")

    def size(self):
        return (self.height, self.r1, self.r2)


class Part:
    """geom::Part: shapes joined by union (add) or difference; the part's
    material (delta, beta)."""

    def __init__(self, name: str = "part", delta: float = 0.0, beta: float = 0.0):
        self.name = name
        self.delta = float(delta)
        self.beta = float(beta)
        self.shapes: List[Shape] = []
        self.operations: List[int] = []

    def add(self, shape: Shape) -> "Part":
        self.shapes.append(shape)
        self.operations.append(UNION)
        return self

    def difference(self, shape: Shape) -> "Part":
        if not self.shapes:
            raise RuntimeError("There is no shape to make difference with. You have to add at "
                               "least one shape before...")
        self.shapes.append(shape)
        self.operations.append(DIFFERENCE)
        return self

    def translate(self, x, y, z):
        for s in self.shapes:
            s.translate(x, y, z)
        return self

    def rotate(self, angle_deg, axis):
        for s in self.shapes:
            s.rotate(angle_deg, axis)
        return self

    def scale(self, factor, axis):
        for s in self.shapes:
            s.scale(factor, axis)
        return self


class Module:
    """geom::Module: parts joined by union (add, the part's material) or
    difference (vacuum)."""

    def __init__(self, name: str = "module"):
        self.name = name
        self.parts: List[Part] = []
        self.operations: List[int] = []

    def add(self, part: Part) -> "Module":
        self.parts.append(part)
        self.operations.append(UNION)
        return self

    def difference(self, part: Part) -> "Module":
        # the reference's condition (src/geometry.cpp:202-210) needs two
        # parts already present
        if len(self.parts) <= 1:
            raise RuntimeError("There have to be at least one part present before making "
                               "difference!")
        self.parts.append(part)
        self.operations.append(DIFFERENCE)
        return self

    def translate(self, x, y, z):
        for p in self.parts:
            p.translate(x, y, z)
        return self

    def rotate(self, angle_deg, axis):
        for p in self.parts:
            p.rotate(angle_deg, axis)
        return self

    def scale(self, factor, axis):
        for p in self.parts:
            p.scale(factor, axis)
        return self


def flatten(modules: Sequence[Module]):
    """(modules, parts, shapes) as plain tuples:
    module (first_part, num_parts); part (operation, first_shape, num_shapes,
    delta, beta); shape (kind, operation, 16 row-major matrix entries, 3 sizes)."""
    mods, parts, shapes = [], [], []
    for m in modules:
        mods.append((len(parts), len(m.parts)))
        for p, pop in zip(m.parts, m.operations):
            parts.append((pop, len(shapes), len(p.shapes), p.delta, p.beta))
            for s, sop in zip(p.shapes, p.operations):
                shapes.append((s.kind, sop, tuple(float(v) for v in s.transformation.reshape(-1)),
                               tuple(s.size())))
    return mods, parts, shapes


def _shape_inside(s: Shape, x: float, y: float, z: float) -> bool:
    tx, ty, tz = s.transform(x, y, z)
    if s.kind == SPHERE:
        return math.sqrt(tx * tx + ty * ty + tz * tz) < s.radius
    if s.kind == BOX:
        Lx, Ly, Lz = s.L
        return (tx > -Lx / 2.0 and tx < Lx / 2.0 and ty > -Ly / 2.0 and ty < Ly / 2.0
                and tz > -Lz / 2.0 and tz < Lz / 2.0)
    h = s.height
    if not (tz < h / 2.0 and tz > -h / 2.0):
        return False
    radius = (s.r2 - s.r1) / h * (tz + h / 2.0) + s.r1
    return math.sqrt(tx * tx + ty * ty) < radius


def part_contains(p: Part, x: float, y: float, z: float) -> bool:
    """geom::Part::isInside: the last shape (scanning backwards) that
    contains the point decides by its operation."""
    for s, op in reversed(list(zip(p.shapes, p.operations))):
        if _shape_inside(s, x, y, z):
            return op == UNION
    return False


def material(modules: Sequence[Module], x: float, y: float, z: float) -> Tuple[float, float]:
    """(delta, beta) at a point by the same rules, in Python (for checks; the
    solvers evaluate on the device)."""
    for m in modules:
        for p, op in reversed(list(zip(m.parts, m.operations))):
            if part_contains(p, x, y, z):
                return (p.delta, p.beta) if op == UNION else (0.0, 0.0)
    return (0.0, 0.0)
