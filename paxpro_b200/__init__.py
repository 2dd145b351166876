"""paxpro_b200 -- B200-native paraxial propagation solvers.

Python face of the C ABI (include/paxpro_b200.h), shaped like the reference's
Solver / ParaxialSimulation API (include/solver.hpp, include/
paraxialSimulation.hpp): a solver is created for a discretised problem, given
a material and an initial field, then stepped; fields come back as numpy
arrays in the reference's layouts (cx_vec for one transverse dimension,
column-major Ny x Nx cx_mat for two).

All compute runs in the CUDA library; importing this package without the
built library raises ImportError.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _capi
from ._capi import (ADI, CRANK_NICHOLSON, FFT_SOLVER_2D, FFT_SOLVER_3D, FP32, FP64,  # noqa: F401
                    PxpError)

_capi.lib()  # fail loudly at import when the CUDA library is absent

KIND_NAMES = {FFT_SOLVER_2D: "FFTSolver2D", CRANK_NICHOLSON: "CrankNicholson",
              FFT_SOLVER_3D: "FFTSolver3D", ADI: "ADI"}


def node_count(mn: float, mx: float, step: float) -> int:
    """ParaxialSimulation::nodeNumber* (src/paraxialSimulation.cpp:107-120)."""
    return int(_capi.lib().pxp_node_count(mn, mx, step))


@dataclass
class Disc:
    """Disctretization record (include/paraxialSimulation.hpp:20-26)."""
    min: float
    max: float
    step: float
    downsampling_ratio: int = 1


@dataclass
class Sphere:
    cx: float
    cy: float
    cz: float
    radius: float
    delta: float
    beta: float


@dataclass
class ProblemSpec:
    kind: int
    x: Disc
    z: Disc
    wavenumber: float
    y: Optional[Disc] = None
    precision: int = FP64
    transparent_bc: bool = False
    absorber_width: float = 0.0
    absorber_damping: float = 0.0
    save_every: int = 0
    device: int = 0

    def to_c(self) -> _capi.Problem:
        p = _capi.Problem()
        p.kind, p.precision = self.kind, self.precision
        for name in ("x", "y", "z"):
            d = getattr(self, name) or self.x
            setattr(p, name, _capi.Discretization(d.min, d.max, d.step, d.downsampling_ratio))
        p.wavenumber = self.wavenumber
        p.transparent_bc = int(self.transparent_bc)
        p.absorber_width, p.absorber_damping = self.absorber_width, self.absorber_damping
        p.save_every, p.device = self.save_every, self.device
        return p


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Solver:
    """One propagation problem resident on the GPU (a C-ABI handle)."""

    def __init__(self, spec: ProblemSpec, keep_initial: bool = False):
        """keep_initial: keep the host initial field given to
        set_initial_conditions, as slice 0 of the post-processing modules'
        field quantities (paxpro_b200.post)."""
        self.spec = spec
        self.keep_initial = keep_initial
        self._u0_host = None
        self._h = C.c_void_p()
        L = _capi.lib()
        _capi.check(L.pxp_solver_create(C.byref(spec.to_c()), C.byref(self._h)))
        nx, ny, nz = C.c_uint(), C.c_uint(), C.c_uint()
        L.pxp_shape(self._h, C.byref(nx), C.byref(ny), C.byref(nz))
        self.nx, self.ny, self.nz = nx.value, ny.value, nz.value
        self.three_d = spec.kind in (FFT_SOLVER_3D, ADI)
        # saved slices of the 3-D solvers: (nx // ratio)^2 block averages
        ratio = max(int(spec.x.downsampling_ratio), 1)
        self.save_n = self.nx // ratio if self.three_d else self.nx

    # -- lifetime
    def close(self) -> None:
        if self._h:
            _capi.lib().pxp_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int) -> None:
        _capi.check(status, self._h)

    @property
    def name(self) -> str:
        return KIND_NAMES[self.spec.kind]

    @property
    def shape(self):
        return (self.ny, self.nx) if self.three_d else (self.nx,)

    # -- material hook
    def set_material_table(self, delta: np.ndarray, beta: np.ndarray) -> None:
        d = np.ascontiguousarray(np.asarray(delta, dtype=np.float64).reshape(-1, order="F"))
        b = np.ascontiguousarray(np.asarray(beta, dtype=np.float64).reshape(-1, order="F"))
        self._check(_capi.lib().pxp_set_material_table(self._h, _dptr(d), _dptr(b), d.size))

    def set_material_planes(self, delta: np.ndarray, beta: np.ndarray, first_step: int,
                            nsteps: int) -> None:
        d = np.ascontiguousarray(delta, dtype=np.float64)
        b = np.ascontiguousarray(beta, dtype=np.float64)
        self._check(_capi.lib().pxp_set_material_planes(self._h, _dptr(d), _dptr(b),
                                                        int(first_step), int(nsteps)))

    def set_material_spheres(self, spheres: Sequence[Sphere]) -> None:
        arr = (_capi.SphereC * max(len(spheres), 1))()
        for i, s in enumerate(spheres):
            arr[i] = _capi.SphereC(s.cx, s.cy, s.cz, s.radius, s.delta, s.beta)
        self._check(_capi.lib().pxp_set_material_spheres(self._h, arr, len(spheres)))

    # -- field
    def set_material_csg(self, modules) -> None:
        """Material from constructive solid geometry (paxpro_b200.csg Modules,
        the reference's CSGMaterial), evaluated on the device."""
        from . import csg as _csg
        mods, parts, shapes = _csg.flatten(modules)
        cm = (_capi.CsgModuleC * max(len(mods), 1))()
        for i, m in enumerate(mods):
            cm[i] = _capi.CsgModuleC(*m)
        cp = (_capi.CsgPartC * max(len(parts), 1))()
        for i, p in enumerate(parts):
            cp[i] = _capi.CsgPartC(*p)
        cs = (_capi.CsgShapeC * max(len(shapes), 1))()
        for i, (kind, op, T, size) in enumerate(shapes):
            cs[i] = _capi.CsgShapeC(kind, op, (C.c_double * 16)(*T), (C.c_double * 3)(*size))
        self._check(_capi.lib().pxp_set_material_csg(self._h, cm, len(mods), cp, len(parts), cs,
                                                     len(shapes)))

    def set_initial_conditions(self, field0: np.ndarray) -> None:
        a = np.asarray(field0, dtype=np.complex128)
        if a.shape != self.shape:
            raise ValueError(f"initial field shape {a.shape} != {self.shape}")
        flat = np.ascontiguousarray(a.reshape(-1, order="F"))
        self._check(_capi.lib().pxp_set_initial_conditions(self._h, _dptr(flat.view(np.float64))))
        self._u0_host = a if self.keep_initial else None

    def set_initial_conditions_device(self, ptr: int) -> None:
        self._check(_capi.lib().pxp_set_initial_conditions_device(self._h, C.c_void_p(ptr)))
        self._u0_host = None

    def step(self, nsteps: int = 1) -> None:
        self._check(_capi.lib().pxp_step(self._h, int(nsteps)))

    def solve(self) -> None:
        self._check(_capi.lib().pxp_solve(self._h))

    def synchronize(self) -> None:
        self._check(_capi.lib().pxp_synchronize(self._h))

    def _unflatten(self, flat: np.ndarray) -> np.ndarray:
        if self.three_d:
            return flat.reshape((self.ny, self.nx), order="F")
        return flat

    def get_last_solution(self) -> np.ndarray:
        out = np.empty(self.nx * self.ny, dtype=np.complex128)
        self._check(_capi.lib().pxp_get_last_solution(self._h, _dptr(out.view(np.float64))))
        return self._unflatten(out)

    def field_device_ptr(self) -> int:
        p = C.c_void_p()
        prec = C.c_int()
        self._check(_capi.lib().pxp_get_field_device(self._h, C.byref(p), C.byref(prec)))
        return p.value

    def stream_ptr(self) -> int:
        """cudaStream_t of the solver (for events / interop)."""
        p = C.c_void_p()
        self._check(_capi.lib().pxp_get_stream(self._h, C.byref(p)))
        return p.value or 0

    def set_initial_conditions_ptr(self, host_ptr: int) -> None:
        """Initial field from host memory at host_ptr (interleaved complex128,
        reference layout); pinned memory makes the copy asynchronous."""
        self._check(_capi.lib().pxp_set_initial_conditions(
            self._h, C.cast(C.c_void_p(host_ptr), C.POINTER(C.c_double))))

    def get_last_solution_ptr(self, host_ptr: int) -> None:
        """Current field into host memory at host_ptr (complex128)."""
        self._check(_capi.lib().pxp_get_last_solution(
            self._h, C.cast(C.c_void_p(host_ptr), C.POINTER(C.c_double))))

    def num_saved(self) -> int:
        c = C.c_int()
        self._check(_capi.lib().pxp_num_saved(self._h, C.byref(c)))
        return c.value

    def get_saved(self, slot: int) -> np.ndarray:
        """Saved field of a save slot; for the 3-D solvers with a transverse
        downsampling ratio r > 1 an (n // r) x (n // r) slice of block
        averages (Solver3D::copyCurrentSolution, src/solver3D.cpp:94-112)."""
        m = self.save_n
        out = np.empty(m * m if self.three_d else m, dtype=np.complex128)
        self._check(_capi.lib().pxp_get_saved(self._h, int(slot), _dptr(out.view(np.float64))))
        return out.reshape((m, m), order="F") if self.three_d else out

    def get_post(self, quantity: int, slot: int = -1) -> np.ndarray:
        """A post-processing quantity (_capi.POST_ABS / POST_ARG / POST_REAL /
        POST_ABS2) of a saved slot, or of the last solution (slot = -1),
        computed on the device."""
        if slot < 0:
            n, shape = self.nx * self.ny, ((self.ny, self.nx) if self.three_d else (self.nx,))
        else:
            m = self.save_n
            n, shape = (m * m, (m, m)) if self.three_d else (m, (m,))
        out = np.empty(n, dtype=np.float64)
        self._check(_capi.lib().pxp_get_post(self._h, int(quantity), int(slot), _dptr(out)))
        return out.reshape(shape, order="F")

    def get_post_resized(self, quantity: int, rows: int, cols: int, slot: int = -1) -> np.ndarray:
        """A post-processing quantity of a 3-D field resized on the device to
        (rows, cols) by resizeMatrix (unchanged unless both shrink)."""
        side = self.nx if slot < 0 else self.save_n
        shape = (rows, cols) if (rows < side and cols < side) else (self.ny if slot < 0 else side, side)
        out = np.empty(shape[0] * shape[1], dtype=np.float64)
        self._check(_capi.lib().pxp_get_post_resized(self._h, int(quantity), int(slot), int(rows),
                                                     int(cols), _dptr(out)))
        return out.reshape(shape, order="F")

    def saved_max_abs(self) -> float:
        """Largest |u| over the filled save slots."""
        v = C.c_double()
        self._check(_capi.lib().pxp_saved_max_abs(self._h, C.byref(v)))
        return v.value

    def farfield(self, pad_length: int = 0, phi_min: float = -90.0, phi_max: float = 90.0,
                 padding: int = _capi.PAD_ZERO, pad_value: complex = 0.0,
                 export_dims: tuple = (0, 0), subtract_reference: bool = False) -> np.ndarray:
        """post::FarField of the last solution, computed on the device: a
        vector for the 2-D kinds, a (rows, cols) matrix for the 3-D kinds
        (see pxp_farfield in include/paxpro_b200.h)."""
        pv = complex(pad_value)
        p = _capi.FarFieldParams(int(pad_length), float(phi_min), float(phi_max), int(padding),
                                 pv.real, pv.imag, int(export_dims[0]), int(export_dims[1]),
                                 1 if subtract_reference else 0)
        r, c = C.c_uint(), C.c_uint()
        self._check(_capi.lib().pxp_farfield_shape(self._h, C.byref(p), C.byref(r), C.byref(c)))
        out = np.empty(r.value * c.value, dtype=np.float64)
        self._check(_capi.lib().pxp_farfield(self._h, C.byref(p), _dptr(out)))
        return out.reshape((r.value, c.value), order="F") if self.three_d else out

    def set_reference(self, field) -> None:
        """The field the 3-D far field subtracts: an array of the solution's
        shape, another Solver (its current field, copied on the device) or
        None to clear."""
        if field is None:
            self._check(_capi.lib().pxp_set_reference(self._h, None))
        elif isinstance(field, Solver):
            self._check(_capi.lib().pxp_set_reference_from(self._h, field._h))
        else:
            a = np.asarray(field, dtype=np.complex128)
            if a.shape != self.shape:
                raise ValueError(f"reference shape {a.shape} != {self.shape}")
            flat = np.ascontiguousarray(a.reshape(-1, order="F"))
            self._check(_capi.lib().pxp_set_reference(self._h, _dptr(flat.view(np.float64))))

    def set_flux_windows(self, first_step: int, start, end) -> None:
        """Per-step index windows [start[k], end[k]] of steps first_step + k
        whose trapezoid sums of |u|^2 the 2-D step kernels compute
        (post::Transmittivity); empty arrays clear them."""
        a = np.ascontiguousarray(np.asarray(start, dtype=np.uint32))
        b = np.ascontiguousarray(np.asarray(end, dtype=np.uint32))
        if a.shape != b.shape or a.ndim != 1:
            raise ValueError("start and end must be 1-D arrays of one length")
        pa = a.ctypes.data_as(C.POINTER(C.c_uint)) if a.size else None
        pb = b.ctypes.data_as(C.POINTER(C.c_uint)) if b.size else None
        self._check(_capi.lib().pxp_set_flux_windows(self._h, int(first_step), int(a.size), pa, pb))

    def get_flux(self, first_step: int, count: int) -> np.ndarray:
        """The trapezoid sums of steps first_step .. first_step + count - 1
        (NaN for steps not run yet)."""
        out = np.empty(count, dtype=np.float64)
        self._check(_capi.lib().pxp_get_flux(self._h, int(first_step), int(count), _dptr(out)))
        return out

    def field_flux(self, start: int, end: int) -> float:
        """Trapezoid sum of |u|^2 of the current field over [start, end]."""
        v = C.c_double()
        self._check(_capi.lib().pxp_field_flux(self._h, int(start), int(end), C.byref(v)))
        return v.value

    def reset(self) -> None:
        self._check(_capi.lib().pxp_reset(self._h))

    def device_bytes(self) -> int:
        b = C.c_size_t()
        self._check(_capi.lib().pxp_device_bytes(self._h, C.byref(b)))
        return b.value

    def get_intensity(self) -> np.ndarray:
        out = np.empty(self.nx * self.ny, dtype=np.float64)
        self._check(_capi.lib().pxp_get_intensity(self._h, _dptr(out)))
        return self._unflatten(out)

    @property
    def current_step(self) -> int:
        s = C.c_uint()
        self._check(_capi.lib().pxp_current_step(self._h, C.byref(s)))
        return s.value


class Batch:
    """Independent solvers advanced together on one device (pxp_batch_*),
    admitted against a device-memory budget."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 150 * 10 ** 9):
        self._b = C.c_void_p()
        _capi.check(_capi.lib().pxp_batch_create(device, hbm_budget_bytes, C.byref(self._b)))
        self._members = {}

    def close(self) -> None:
        if self._b:
            _capi.lib().pxp_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, solver: "Solver", nsteps: int) -> bool:
        """True when admitted; False when the memory budget is full."""
        rc = _capi.lib().pxp_batch_admit(self._b, solver._h, int(nsteps))
        if rc == _capi.PXP_ERR_NOT_READY:
            return False
        _capi.check(rc)
        self._members[solver._h.value] = solver
        return True

    def round(self, max_steps: int) -> None:
        _capi.check(_capi.lib().pxp_batch_round(self._b, int(max_steps)))

    def collect(self) -> list:
        cap = max(len(self._members), 1)
        arr = (C.c_void_p * cap)()
        cnt = C.c_int()
        _capi.check(_capi.lib().pxp_batch_collect(self._b, arr, cap, C.byref(cnt)))
        return [self._members.pop(arr[i]) for i in range(cnt.value)]

    def status(self):
        a, b = C.c_int(), C.c_size_t()
        _capi.check(_capi.lib().pxp_batch_status(self._b, C.byref(a), C.byref(b)))
        return a.value, b.value


__all__ = ["Batch", "Solver", "ProblemSpec", "Disc", "Sphere", "node_count", "PxpError",
           "FFT_SOLVER_2D", "CRANK_NICHOLSON", "FFT_SOLVER_3D", "ADI", "FP64", "FP32"]
