"""Synthetic workloads with the shapes and value distributions of the
benchmark configurations.

All lengths are in nm; wavelength 0.1 nm (k = 2 pi / 0.1).  Randomness uses
numpy.random.default_rng(seed).  The reference publishes no input files for
these problems, so every input here is generated.

  waveguide_2d   planar waveguide: vacuum core |x| <= w, cladding (delta,
                 beta) elsewhere, and a linear beta ramp to 1e-4 over the 25
                 outermost grid points on each side standing in for an
                 absorbing boundary (the reference's 2-D solvers have none;
                 Examples/waveguide2D.cpp:9-31 shows the material-function
                 pattern).
  waveguide_fft2d  FFTSolver2D, Nx = 2048 on [-250, 250], 4000 steps of 1 um,
                   Gaussian waist 15 nm, saves every 100 steps.
  waveguide_cn     CrankNicholson, Nx = 4096, 8000 steps of 0.5 um, same guide.
  sphere_adi       ADI, 1024^2 on [-500, 500]^2, 2000 steps of 1 um, unit plane
                   wave, sphere R = 200 at (0, 0, 1 mm).
  spheres_fft3d    FFTSolver3D, 4096^2 on [-1000, 1000]^2, 1000 steps of 2 um,
                   unit plane wave, 64 seeded spheres.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

WAVELENGTH = 0.1
K = 2.0 * math.acos(-1.0) / WAVELENGTH  # ParaxialSimulation::setWaveLength


def node_count(mn: float, mx: float, step: float) -> int:
    """Truncating node count of src/paraxialSimulation.cpp:107-120."""
    return int((mx - mn) / step + 1.0)


def step_for_nodes(mn: float, mx: float, n: int) -> float:
    """A step for which the reference's node-count expression gives exactly n."""
    step = (mx - mn) / (n - 1)
    for _ in range(64):
        c = node_count(mn, mx, step)
        if c == n:
            return step
        step = np.nextafter(step, 0.0 if c < n else np.inf)
    raise ValueError("no step gives the requested node count")


def coords(mn: float, step: float, n: int) -> np.ndarray:
    """ParaxialSimulation::getX (src/paraxialSimulation.cpp:255-258)."""
    return mn + np.arange(n, dtype=np.float64) * step


@dataclass
class Waveguide:
    core_half_width: float = 25.0
    delta_clad: float = 7.5e-6
    beta_clad: float = 1.0e-7
    ramp_points: int = 25
    ramp_beta: float = 1.0e-4

    def tables(self, x: np.ndarray):
        """delta/beta per grid point (index-based ramp, then core/cladding)."""
        n = len(x)
        ix = np.arange(n)
        d = np.minimum(ix, n - 1 - ix)
        delta = np.where(np.abs(x) <= self.core_half_width, 0.0, self.delta_clad)
        beta = np.where(np.abs(x) <= self.core_half_width, 0.0, self.beta_clad)
        ramp = d < self.ramp_points
        rb = self.beta_clad + (self.ramp_beta - self.beta_clad) * \
            (self.ramp_points - d).astype(np.float64) / float(self.ramp_points)
        delta = np.where(ramp, self.delta_clad, delta)
        beta = np.where(ramp, rb, beta)
        return delta.astype(np.float64), beta.astype(np.float64)


@dataclass
class Problem2D:
    name: str
    kind: str  # "fft" | "cn"
    xmin: float
    xmax: float
    dx: float
    zmin: float
    zmax: float
    dz: float
    nsteps: int
    waist: float
    guide: Waveguide
    save_every: int = 100
    center: float = 0.0

    @property
    def nx(self) -> int:
        return node_count(self.xmin, self.xmax, self.dx)

    @property
    def x(self) -> np.ndarray:
        return coords(self.xmin, self.dx, self.nx)

    def initial_field(self) -> np.ndarray:
        """GaussianBeam at z = z0 = 0: exp(-((x - xc)/w)^2), zero phase
        (src/gaussianBeam.cpp:29-40 at z = 0)."""
        x = self.x - self.center
        return np.exp(-(x / self.waist) ** 2).astype(np.complex128)

    def material(self):
        return self.guide.tables(self.x)


@dataclass
class Problem3D:
    name: str
    kind: str  # "fft3d" | "adi"
    xmin: float
    xmax: float
    dx: float
    zmin: float
    zmax: float
    dz: float
    nsteps: int
    spheres: List[tuple] = field(default_factory=list)  # (cx, cy, cz, R, delta, beta)
    save_every: int = 100

    @property
    def nx(self) -> int:
        return node_count(self.xmin, self.xmax, self.dx)

    def initial_field(self) -> np.ndarray:
        """Unit plane wave at normal incidence (PlaneWave::get, src/planeWave.cpp:5-14)."""
        n = self.nx
        return np.ones((n, n), dtype=np.complex128, order="F")


def waveguide_fft2d(nsteps: int = 4000) -> Problem2D:
    xmin, xmax = -250.0, 250.0
    return Problem2D("waveguide_fft2d", "fft", xmin, xmax, step_for_nodes(xmin, xmax, 2048),
                     0.0, 4.0e6, 1000.0, nsteps, 15.0, Waveguide())


def waveguide_cn(nsteps: int = 8000) -> Problem2D:
    xmin, xmax = -250.0, 250.0
    return Problem2D("waveguide_cn", "cn", xmin, xmax, step_for_nodes(xmin, xmax, 4096),
                     0.0, 4.0e6, 500.0, nsteps, 15.0, Waveguide())


def sphere_adi(nsteps: int = 2000, n: int = 1024) -> Problem3D:
    xmin, xmax = -500.0, 500.0
    return Problem3D("sphere_adi", "adi", xmin, xmax, step_for_nodes(xmin, xmax, n),
                     0.0, 2.0e6, 1000.0, nsteps,
                     [(0.0, 0.0, 1.0e6, 200.0, 4.5e-5, 3.6e-6)])


def random_spheres(rng: np.random.Generator, count: int, lo: float, hi: float, zmax: float):
    out = []
    for _ in range(count):
        r = rng.uniform(20.0, 150.0)
        cx, cy = rng.uniform(lo, hi), rng.uniform(lo, hi)
        cz = rng.uniform(0.0, zmax)
        delta = rng.uniform(1e-6, 5e-5)
        out.append((cx, cy, cz, r, delta, delta / 50.0))
    return out


def spheres_fft3d(nsteps: int = 1000, n: int = 4096, seed: int = 2) -> Problem3D:
    xmin, xmax = -1000.0, 1000.0
    rng = np.random.default_rng(seed)
    return Problem3D("spheres_fft3d", "fft3d", xmin, xmax, step_for_nodes(xmin, xmax, n),
                     0.0, 2.0e6, 2000.0, nsteps, random_spheres(rng, 64, xmin, xmax, 2.0e6))
