"""GenericScattering: a Gaussian beam through a 3-D object, on the device.

The reference's application class (include/genericScattering.hpp:11-87,
src/genericScattering.cpp) with its public fields: a reference run in vacuum
over the same z range in three steps (init, :21-135), whose exit field the
far field subtracts (:160-178), then the run through the object with the
user's dz (:181-212); the far field (post::FarField, computed on the device)
resized to exportNx x exportNy, and the exit field, intensity and phase.

The object is a sphere list (paxpro_b200.Sphere) or constructive solid
geometry (paxpro_b200.csg Modules), both evaluated by the solvers on the
device.  With the ADI propagator any node count runs; FFTSolver3D needs a
power of two per transverse axis.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import _capi
from .sources import GaussianBeam


class GenericScattering:
    ADI, FFT = "adi", "fft"

    def __init__(self, name: str = "GenericScattering"):
        self.name = name
        self.description = ""
        self.exportNx = 512
        self.exportNy = 512
        self.FFTPadLength = 1024
        self.xmin, self.xmax = -1.0, 1.0
        self.ymin, self.ymax = -1.0, 1.0
        self.zmin, self.zmax = -1.0, 1.0
        self.dx = self.dy = self.dz = 0.1
        self.downSampleZ = 1
        self.wavelength = 0.1569
        self.subtract_reference = True
        self.propagator = self.FFT
        self.precision = _capi.FP64
        self._beam = GaussianBeam()
        self._phi = (-90.0, 90.0)
        self._material = None
        self.reference: Optional[np.ndarray] = None
        self.exit_field: Optional[np.ndarray] = None
        self._solver = None

    def setBeamWaist(self, waist: float) -> None:
        self._beam.waist = float(waist)

    def setMaxScatteringAngle(self, angle: float) -> None:
        """FarField::setAngleRange(-angle, angle) (src/genericScattering.cpp:16-19)."""
        self._phi = (-float(angle), float(angle))

    def setMaterial(self, material) -> None:
        """A list of paxpro_b200.Sphere, or of paxpro_b200.csg.Module."""
        self._material = material

    def _spec(self, dz: float, save_every: int):
        from . import Disc, ProblemSpec
        kind = _capi.ADI if self.propagator == self.ADI else _capi.FFT_SOLVER_3D
        k = 2.0 * np.pi / self.wavelength
        # ADI::useTBC defaults to true (include/alternatingDirectionSolver.hpp:24)
        return ProblemSpec(kind=kind, x=Disc(self.xmin, self.xmax, self.dx),
                           y=Disc(self.ymin, self.ymax, self.dy),
                           z=Disc(self.zmin, self.zmax, dz), wavenumber=k,
                           precision=self.precision, save_every=save_every,
                           transparent_bc=kind == _capi.ADI)

    def _initial(self) -> np.ndarray:
        from . import node_count
        self._beam.set_wavelength(self.wavelength)
        nx = node_count(self.xmin, self.xmax, self.dx)
        ny = node_count(self.ymin, self.ymax, self.dy)
        x = self.xmin + self.dx * np.arange(nx)
        y = self.ymin + self.dy * np.arange(ny)
        return self._beam.field_3d(x, y)

    def _apply_material(self, solver) -> None:
        from . import Sphere
        from .csg import Module
        m = self._material
        if m and all(isinstance(v, Sphere) for v in m):
            solver.set_material_spheres(list(m))
        elif m and all(isinstance(v, Module) for v in m):
            solver.set_material_csg(list(m))
        else:
            raise TypeError("the material must be a list of Sphere or of csg.Module")

    def solve(self) -> None:
        """GenericScattering::solve (src/genericScattering.cpp:148-213)."""
        from . import Solver
        if not self._material:
            raise RuntimeError("No material set!")
        self.close()
        u0 = self._initial()
        with Solver(self._spec((self.zmax - self.zmin) / 3.0, 0)) as ref:
            ref.set_initial_conditions(u0)
            ref.solve()
            self.reference = ref.get_last_solution()
            s = Solver(self._spec(self.dz, self.downSampleZ))
            try:
                self._apply_material(s)
                s.set_initial_conditions(u0)
                s.solve()
                if self.subtract_reference:
                    s.set_reference(ref)   # device-to-device copy
            except Exception:
                s.close()
                raise
        self._solver = s
        self.exit_field = s.get_last_solution()

    @property
    def solver(self):
        return self._solver

    def getFarField(self) -> np.ndarray:
        """post::FarField of the exit field (minus the reference run's),
        resized to exportNx x exportNy (src/genericScattering.cpp:235-238)."""
        if self._solver is None:
            raise RuntimeError("solve() first")
        return self._solver.farfield(pad_length=self.FFTPadLength, phi_min=self._phi[0],
                                     phi_max=self._phi[1], export_dims=(self.exportNx, self.exportNy),
                                     subtract_reference=self.subtract_reference)

    def modules(self):
        """The modules GenericScattering attaches (src/genericScattering.cpp:
        28-33, 121): ExitField, ExitIntensity, ExitPhase and FarField, each
        with the export dimensions."""
        from . import post
        mods = [post.ExitField(), post.ExitIntensity(), post.ExitPhase(),
                post.FarField(self.FFTPadLength, self._phi[0], self._phi[1],
                              subtract_reference=self.subtract_reference)]
        for m in mods:
            m.set_export_dimensions(self.exportNx, self.exportNy)
        return mods

    def save(self, path: str):
        """The datasets ParaxialSimulation::save writes for this simulation,
        as .npy files (see paxpro_b200.post.save)."""
        from . import post
        if self._solver is None:
            raise RuntimeError("solve() first")
        return post.save(self._solver, path, self.modules(), self.description)

    def close(self) -> None:
        if self._solver is not None:
            self._solver.close()
            self._solver = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
