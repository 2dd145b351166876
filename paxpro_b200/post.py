"""Post-processing modules and the save path of a simulation.

The reference's post:: modules (src/postProcessMod.cpp:7-150,
include/postProcessMod.hpp) turn a solver's stored fields into the datasets
`ParaxialSimulation::save` writes (src/paraxialSimulation.cpp:137-193):

  * field quantities over every stored slice -- `Intensity` ("amplitude",
    |u|), `IntensityUint8` ("amplitude", 255 |u| / max |u|),
    `LogIntensityUint8` ("LogAmplitude"), `Phase` ("phase", arg u): a matrix
    (points x slices) for the 2-D solvers, a cube (rows x cols x slices) for
    the 3-D solvers;
  * projection quantities of the exit field -- `ExitField` ("exitField",
    Re u), `ExitIntensity` ("exitIntensity", |u|^2), `ExitPhase`
    ("exitPhase", arg u): a vector (2-D) or a matrix (3-D), resized on the
    device after set_export_dimensions; `FarField` ("farField").

The stored slices are the initial condition (slice 0, from the host copy the
solver keeps when it was given a host array) followed by the saved fields
(every `save_every` steps; the reference's 2-D solvers keep every step, its
3-D solvers every longitudinal-ratio steps).  The per-point reductions of
saved fields and of the exit field run on the device (`pxp_get_post`): only
8 bytes per point come back.

`save` writes the datasets under the reference's names: HDF5 is not
available here, so `<path>/data/<name>.npy` (column-major arrays, as
Armadillo stores them) plus `<path>/data/attributes.json` with the group
attributes of `ParaxialSimulation::setGroupAttributes`
(src/paraxialSimulation.cpp:453-510).
"""
from __future__ import annotations

import json
import math
import os
from typing import Iterable, List, Optional

import numpy as np

from . import _capi

SOLVER_NAMES = {_capi.FFT_SOLVER_2D: "FFTSolver2D", _capi.CRANK_NICHOLSON: "CrankNicholson",
                _capi.FFT_SOLVER_3D: "FFTSolver3D", _capi.ADI: "ADI"}


def _block_average(u: np.ndarray, m: int) -> np.ndarray:
    """Solver3D::copyCurrentSolution's block average (src/solver3D.cpp:94-112)
    of the n x n initial field to m x m (slice 0 of a downsampled cube)."""
    n = u.shape[0]
    if m == n:
        return u
    delta = n / m
    out = np.empty((m, m), dtype=np.complex128)
    for col in range(m):
        c0, c1 = int(col * delta), int(col * delta + delta - 1)
        for row in range(m):
            r0, r1 = int(row * delta), int(row * delta + delta - 1)
            out[row, col] = u[r0:r1 + 1, c0:c1 + 1].sum(axis=0).sum() / (delta * delta)
    return out


class PostProcessingModule:
    name = ""
    is_uint8 = False
    export_dims = None

    def set_export_dimensions(self, rows: int, cols: int) -> None:
        """PostProcessingModule::setExportDimensions (src/postProcessing.cpp:51-56):
        3-D projection results are resized by resizeMatrix (:29-49), on the
        device, when both dimensions are smaller."""
        self.export_dims = (int(rows), int(cols))

    def result(self, solver) -> np.ndarray:
        raise NotImplementedError


class FieldQuantity(PostProcessingModule):
    """A quantity over every stored slice (post::FieldQuantity)."""

    quantity = _capi.POST_ABS

    def _host(self, u: np.ndarray) -> np.ndarray:
        return np.abs(u) if self.quantity == _capi.POST_ABS else np.angle(u)

    def slices(self, solver) -> List[np.ndarray]:
        out = []
        u0 = getattr(solver, "_u0_host", None)
        if u0 is not None:
            out.append(self._host(_block_average(u0, solver.save_n) if solver.three_d else u0))
        for k in range(solver.num_saved()):
            out.append(solver.get_post(self.quantity, k))
        return out

    def result(self, solver) -> np.ndarray:
        s = self.slices(solver)
        return np.stack(s, axis=-1) if s else np.empty((0,))


class Intensity(FieldQuantity):
    """|u| of every stored slice (post::Intensity, src/postProcessMod.cpp:7-15)."""
    name = "amplitude"
    quantity = _capi.POST_ABS


class Phase(FieldQuantity):
    """arg u of every stored slice (post::Phase, src/postProcessMod.cpp:86-100)."""
    name = "phase"
    quantity = _capi.POST_ARG


class IntensityUint8(FieldQuantity):
    """255 |u| / max |u| over the whole cube, truncated to 8 bits
    (post::IntensityUint8, src/postProcessMod.cpp:17-30)."""
    name = "amplitude"
    quantity = _capi.POST_ABS
    is_uint8 = True

    def result(self, solver) -> np.ndarray:
        a = super().result(solver)
        m = float(a.max()) if a.size else 0.0
        return np.trunc(255.0 * a / m).astype(np.uint8)


class LogIntensityUint8(FieldQuantity):
    """255 (log|u| - min) / (max - min), clamped to [0, 255], with min / max
    the log of the smallest / largest |u| or the set limits
    (post::LogIntensityUint8, src/postProcessMod.cpp:32-84)."""
    name = "LogAmplitude"
    quantity = _capi.POST_ABS
    is_uint8 = True

    def __init__(self):
        self.minval: Optional[float] = None
        self.maxval: Optional[float] = None

    def set_min_value(self, v: float) -> None:
        self.minval = math.log(v)

    def set_max_value(self, v: float) -> None:
        self.maxval = math.log(v)

    def result(self, solver) -> np.ndarray:
        a = super().result(solver)
        with np.errstate(divide="ignore"):
            la = np.log(a)
        hi, lo = float(la.max()), float(la.min())
        hi = min(self.maxval, hi) if self.maxval is not None else hi
        lo = max(self.minval, lo) if self.minval is not None else lo
        with np.errstate(invalid="ignore"):
            mid = np.trunc(255.0 * (la - lo) / (hi - lo))
        out = np.where(la > hi, 255.0, np.where(la < lo, 0.0, mid))
        return out.astype(np.uint8)


class ProjectionQuantity(PostProcessingModule):
    """A quantity of the exit field (post::ProjectionQuantity)."""

    quantity = _capi.POST_REAL

    def result(self, solver) -> np.ndarray:
        if solver.three_d and self.export_dims:
            return solver.get_post_resized(self.quantity, *self.export_dims)
        return solver.get_post(self.quantity, -1)


class ExitField(ProjectionQuantity):
    """Re u of the exit field (post::ExitField, src/postProcessMod.cpp:102-116)."""
    name = "exitField"
    quantity = _capi.POST_REAL


class ExitIntensity(ProjectionQuantity):
    """pow(|u|, 2) of the exit field (post::ExitIntensity, :118-132)."""
    name = "exitIntensity"
    quantity = _capi.POST_ABS2


class ExitPhase(ProjectionQuantity):
    """arg u of the exit field (post::ExitPhase, :134-150)."""
    name = "exitPhase"
    quantity = _capi.POST_ARG


class FarField(ProjectionQuantity):
    """post::FarField (src/farFieldPost.cpp): |FFT| of the padded exit field
    (2-D) or the |.|^2 / L of the two padded transforms of the exit field
    minus a reference (3-D), over the angular window, computed on the
    device by Solver.farfield."""
    name = "farField"

    def __init__(self, pad_length: int = 0, phi_min: float = -90.0, phi_max: float = 90.0,
                 padding: int = _capi.PAD_ZERO, pad_value: complex = 0.0,
                 subtract_reference: bool = False):
        self.pad_length = pad_length
        self.phi = (phi_min, phi_max)
        self.padding = padding
        self.pad_value = pad_value
        self.subtract_reference = subtract_reference

    def set_angle_range(self, phi_min: float, phi_max: float) -> None:
        self.phi = (float(phi_min), float(phi_max))

    def attributes(self, solver) -> dict:
        """FarField::addAttrib (src/farFieldPost.cpp:131-139)."""
        k = solver.spec.wavenumber
        return {"phiMin": self.phi[0], "phiMax": self.phi[1],
                "qmin": self.phi[0] * k * math.pi / 180.0, "qmax": self.phi[1] * k * math.pi / 180.0}

    def result(self, solver) -> np.ndarray:
        return solver.farfield(pad_length=self.pad_length, phi_min=self.phi[0],
                               phi_max=self.phi[1], padding=self.padding, pad_value=self.pad_value,
                               export_dims=self.export_dims or (0, 0),
                               subtract_reference=self.subtract_reference)


def group_attributes(solver, description: str = "") -> dict:
    """ParaxialSimulation::setGroupAttributes (src/paraxialSimulation.cpp:453-510)."""
    sp = solver.spec
    y = sp.y if solver.three_d else sp.x
    attrs = {"xmin": sp.x.min, "xmax": sp.x.max, "dx": sp.x.step,
             "zmin": sp.z.min, "zmax": sp.z.max, "dz": sp.z.step,
             "ymin": y.min, "ymax": y.max, "dy": y.step,
             "wavenumber": sp.wavenumber, "solver": SOLVER_NAMES.get(sp.kind, "")}
    if description:
        attrs["description"] = description
    return attrs


def save(solver, path: str, modules: Iterable[PostProcessingModule], description: str = "") -> List[str]:
    """Write every module's result as `<path>/data/<name>.npy` (column-major,
    as Armadillo stores it) and the group attributes as
    `<path>/data/attributes.json`; returns the dataset paths written.  A later
    module with the same name replaces an earlier one, as a second HDF5
    dataset of that name could not be created."""
    d = os.path.join(path, "data")
    os.makedirs(d, exist_ok=True)
    written = []
    for mod in modules:
        arr = np.asfortranarray(mod.result(solver))
        f = os.path.join(d, mod.name + ".npy")
        np.save(f, arr)
        written.append(f)
    attrs = group_attributes(solver, description)
    for mod in modules:
        extra = getattr(mod, "attributes", None)
        if extra is not None:
            attrs[mod.name] = extra(solver)
    with open(os.path.join(d, "attributes.json"), "w") as fh:
        json.dump(attrs, fh, indent=1, sort_keys=True)
    return written
