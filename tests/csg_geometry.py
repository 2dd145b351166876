"""A constructive-solid-geometry test material: two modules, unions and
differences at both levels, rotated, translated and scaled shapes of all
three kinds, placed across the sampling planes z = 3000, 4000, 5000, 6000.

The scene is written once as data (SCENE) and built from it two ways:
`geometry()` gives the paxpro_b200.csg objects the solvers take, and
`reference_arrays()` the description oracle/_ref's ref_csg_eval builds the
reference's own geom:: objects from, replaying the same transform calls in
the same order."""
import ctypes as C

from paxpro_b200 import csg

# module -> parts (operation, delta, beta, shapes); shape (operation, kind and
# sizes, transform calls in order)
SCENE = [
    [  # "lens"
        ("add", 3e-5, 6e-7, [
            ("add", ("box", 300.0, 200.0, 150.0), [("rotate", 30.0, csg.Z),
                                                   ("translate", 0.0, 0.0, 3000.0)]),
            ("difference", ("sphere", 60.0), [("translate", 20.0, 0.0, 3000.0)]),
        ]),
        ("add", 1e-5, 2e-7, [
            ("add", ("cylinder", 40.0, 80.0, 400.0), [("rotate", 90.0, csg.X),
                                                       ("translate", -150.0, 50.0, 5000.0)]),
        ]),
    ],
    [  # "shell"
        ("add", 2e-5, 4e-7, [("add", ("sphere", 120.0), [("translate", 100.0, -100.0, 4000.0)])]),
        ("add", 5e-6, 1e-7, [("add", ("sphere", 50.0), [("scale", 2.0, csg.Z),
                                                         ("translate", -300.0, 300.0, 6000.0)])]),
        ("difference", 9e-5, 9e-7, [("add", ("box", 50.0, 50.0, 50.0),
                                     [("translate", 100.0, -100.0, 4000.0)])]),
    ],
]


def _shape(desc):
    kind, *size = desc
    if kind == "sphere":
        return csg.Sphere(*size)
    if kind == "box":
        return csg.Box(*size)
    return csg.Cylinder(*size)


def geometry(scene=SCENE):
    modules = []
    for parts in scene:
        mod = csg.Module()
        for op, delta, beta, shapes in parts:
            part = csg.Part(delta=delta, beta=beta)
            for sop, desc, calls in shapes:
                s = _shape(desc)
                for call, *args in calls:
                    getattr(s, call)(*args)
                part.add(s) if sop == "add" else part.difference(s)
            mod.add(part) if op == "add" else mod.difference(part)
        modules.append(mod)
    return modules


class RefShape(C.Structure):
    _fields_ = [("kind", C.c_int), ("operation", C.c_int), ("first_op", C.c_int),
                ("num_ops", C.c_int), ("size", C.c_double * 3)]


class RefOp(C.Structure):
    _fields_ = [("type", C.c_int), ("a", C.c_double), ("b", C.c_double), ("c", C.c_double)]


class RefPart(C.Structure):
    _fields_ = [("operation", C.c_int), ("first_shape", C.c_int), ("num_shapes", C.c_int),
                ("delta", C.c_double), ("beta", C.c_double)]


class RefModule(C.Structure):
    _fields_ = [("first_part", C.c_int), ("num_parts", C.c_int)]


def reference_arrays(scene=SCENE):
    """(modules, parts, shapes, ops) ctypes arrays for ref_csg_eval."""
    kinds = {"sphere": 0, "box": 1, "cylinder": 2}
    calls_t = {"translate": 0, "rotate": 1, "scale": 2}
    mods, parts, shapes, ops = [], [], [], []
    for mparts in scene:
        mods.append(RefModule(len(parts), len(mparts)))
        for op, delta, beta, pshapes in mparts:
            parts.append(RefPart(0 if op == "add" else 1, len(shapes), len(pshapes), delta, beta))
            for sop, desc, calls in pshapes:
                kind, *size = desc
                size = list(size) + [0.0] * (3 - len(size))
                shapes.append(RefShape(kinds[kind], 0 if sop == "add" else 1, len(ops), len(calls),
                                       (C.c_double * 3)(*size)))
                for call, *args in calls:
                    args = [float(a) for a in args] + [0.0] * (3 - len(args))
                    ops.append(RefOp(calls_t[call], *args))
    return ((RefModule * len(mods))(*mods), (RefPart * len(parts))(*parts),
            (RefShape * len(shapes))(*shapes), (RefOp * max(len(ops), 1))(*ops))
