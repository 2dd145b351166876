"""Initial fields of a simulation: the reference's paraxial sources.

GaussianBeam (include/gaussianBeam.hpp, src/gaussianBeam.cpp:7-63) and
PlaneWave (src/planeWave.cpp:5-19), evaluated on the grid at z = 0 the way
ParaxialSimulation::setBoundaryConditions does (src/paraxialSimulation.cpp:
356-399): a vector over x for 2-D solvers, an (Ny, Nx) matrix (rows y,
columns x, Fortran order) for 3-D solvers.  Each point follows the
reference's expression term by term in FP64.
"""
from __future__ import annotations

import math

import numpy as np

PI = math.acos(-1.0)


class ParaxialSource:
    def __init__(self):
        self.wavenumber = 0.0
        self.z0 = 0.0
        self.amplitude = 1.0

    def set_wavelength(self, wavelength: float) -> None:
        self.wavenumber = 2.0 * PI / wavelength

    @property
    def wavelength(self) -> float:
        return 2.0 * PI / self.wavenumber

    def field_2d(self, x: np.ndarray) -> np.ndarray:
        return np.array([self.get(float(v), 0.0) for v in x], dtype=np.complex128)

    def field_3d(self, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        out = np.empty((y.size, x.size), dtype=np.complex128, order="F")
        for i, xv in enumerate(x):
            for j, yv in enumerate(y):
                out[j, i] = self.get3(float(xv), float(yv), 0.0)
        return out


class GaussianBeam(ParaxialSource):
    def __init__(self, waist: float = 1.0):
        super().__init__()
        self.waist = float(waist)
        self.center_x = 0.0
        self.center_y = 0.0
        self.angle_x = 0.0
        self.angle_y = 0.0

    def _zr(self):
        return PI * self.waist * self.waist / self.wavelength

    def _spot(self, z):
        return self.waist * math.sqrt(1.0 + (z / self._zr()) ** 2)

    def _inv_r(self, z):
        zr = self._zr()
        return z / (z * z + zr * zr)

    def _angle(self, deg, x):
        return complex(math.cos(self.wavenumber * math.sin(deg * PI / 180.0) * x),
                       math.sin(self.wavenumber * math.sin(deg * PI / 180.0) * x))

    def get(self, x: float, z: float) -> complex:
        """GaussianBeam::get(x, z) (src/gaussianBeam.cpp:29-39)."""
        x -= self.center_x
        dz = z - self.z0
        waist_ratio = self.waist / self._spot(dz)
        gaussian = math.exp(-((x / self._spot(dz)) ** 2))
        ph = (-self.wavenumber * self.z0 + 0.5 * self.wavenumber * x * x * self._inv_r(dz)
              - math.atan(dz / self._zr()))
        phase = complex(math.cos(ph), math.sin(ph))
        return self.amplitude * waist_ratio * gaussian * phase * self._angle(self.angle_x, x)

    def get3(self, x: float, y: float, z: float) -> complex:
        """GaussianBeam::get(x, y, z) (:57-63)."""
        y -= self.center_y
        gauss_y = math.exp(-((y / self._spot(z - self.z0)) ** 2))
        return self.get(x, z) * gauss_y * self._angle(self.angle_y, y)


class PlaneWave(ParaxialSource):
    def __init__(self, angle_deg: float = 0.0):
        super().__init__()
        self.angle = angle_deg * PI / 180.0

    def get(self, x: float, z: float) -> complex:
        ph = self.wavenumber * x * math.sin(self.angle) - self.wavenumber * self.z0
        return self.amplitude * complex(math.cos(ph), math.sin(ph))

    def get3(self, x: float, y: float, z: float) -> complex:
        return self.get(x, z)
