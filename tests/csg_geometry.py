"""A constructive-solid-geometry test material: two modules, unions and
differences at both levels, rotated, translated and scaled shapes of all
three kinds, placed across the sampling planes z = 3000, 4000, 5000, 6000."""
from paxpro_b200 import csg


def geometry():
    lens = csg.Module("lens")
    p1 = csg.Part("slab", delta=3e-5, beta=6e-7)
    p1.add(csg.Box(300.0, 200.0, 150.0).rotate(30.0, csg.Z).translate(0.0, 0.0, 3000.0))
    p1.difference(csg.Sphere(60.0).translate(20.0, 0.0, 3000.0))
    p2 = csg.Part("cone", delta=1e-5, beta=2e-7)
    p2.add(csg.Cylinder(40.0, 80.0, 400.0).rotate(90.0, csg.X).translate(-150.0, 50.0, 5000.0))
    lens.add(p1).add(p2)
    shell = csg.Module("shell")
    p3 = csg.Part("ball", delta=2e-5, beta=4e-7)
    p3.add(csg.Sphere(120.0).translate(100.0, -100.0, 4000.0))
    p5 = csg.Part("far", delta=5e-6, beta=1e-7)
    p5.add(csg.Sphere(50.0).scale(2.0, csg.Z).translate(-300.0, 300.0, 6000.0))
    p4 = csg.Part("hole", delta=9e-5, beta=9e-7)
    p4.add(csg.Box(50.0, 50.0, 50.0).translate(100.0, -100.0, 4000.0))
    shell.add(p3).add(p5).difference(p4)
    return [lens, shell]
