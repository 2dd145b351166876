"""ctypes front end to the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline leg, never by the product package.  Arrays are numpy complex128;
2-transverse-dim fields are (Ny, Nx) arrays stored Fortran-order so that the
memory layout is the reference's Armadillo column-major cx_mat.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REFPIN = None


class Grid(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "xmin", "xmax", "dx", "ymin", "ymax", "dy", "zmin", "zmax", "dz",
        "wavenumber")]


class Sphere(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("cx", "cy", "cz", "radius", "delta", "beta")]


class Material(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("core_half_width", C.c_double), ("delta_clad", C.c_double),
        ("beta_clad", C.c_double), ("ramp_beta", C.c_double),
        ("ramp_points", C.c_int), ("n_transverse", C.c_int),
        ("spheres", C.POINTER(Sphere)), ("n_spheres", C.c_int),
        ("delta_table", C.POINTER(C.c_double)), ("beta_table", C.POINTER(C.c_double)),
        ("csg_modules", C.c_void_p), ("n_csg_modules", C.c_int),
        ("csg_parts", C.c_void_p), ("csg_shapes", C.c_void_p),
    ]


class CsgShape(C.Structure):
    _fields_ = [("kind", C.c_int), ("operation", C.c_int), ("transform", C.c_double * 16),
                ("size", C.c_double * 3)]


class CsgPart(C.Structure):
    _fields_ = [("operation", C.c_int), ("first_shape", C.c_int), ("num_shapes", C.c_int),
                ("delta", C.c_double), ("beta", C.c_double)]


class CsgModule(C.Structure):
    _fields_ = [("first_part", C.c_int), ("num_parts", C.c_int)]


MAT_VACUUM, MAT_WAVEGUIDE, MAT_SPHERES, MAT_XTABLE, MAT_CSG = 0, 1, 2, 3, 4


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        d = C.POINTER(C.c_double)
        _LIB.orc_node_count.restype = C.c_uint
        _LIB.orc_node_count.argtypes = [C.c_double] * 3
        _LIB.orc_fft1d.argtypes = [d, C.c_int, C.c_int]
        _LIB.orc_thomas.argtypes = [d, d, d, C.c_int]
        _LIB.orc_block_average.argtypes = [d, C.c_int, C.c_int, d]
        _LIB.orc_block_average.restype = None
        for name in ("orc_fft2d_run",):
            getattr(_LIB, name).argtypes = [C.POINTER(Grid), C.POINTER(Material), d,
                                            C.c_int, C.c_int, d, d]
        for name in ("orc_cn2d_run", "orc_adi3d_run"):
            getattr(_LIB, name).argtypes = [C.POINTER(Grid), C.POINTER(Material), C.c_int,
                                            d, C.c_int, C.c_int, d, d]
        _LIB.orc_fft3d_run.argtypes = [C.POINTER(Grid), C.POINTER(Material), C.c_double,
                                       C.c_double, d, C.c_int, C.c_int, d, d]
        _LIB.orc_gaussian_beam_2d.argtypes = [C.POINTER(Grid)] + [C.c_double] * 5 + [d]
        _LIB.orc_gaussian_beam_3d.argtypes = [C.POINTER(Grid)] + [C.c_double] * 6 + [d]
        _LIB.orc_material_eval.argtypes = [C.POINTER(Material), C.POINTER(Grid)] + \
            [C.c_double] * 3 + [d, d]
        _LIB.orc_set_threads.argtypes = [C.c_int]
        _LIB.orc_material_planes.argtypes = [C.POINTER(Grid), C.POINTER(Material), C.c_int,
                                             C.c_int, C.c_int, d, d]
        _LIB.orc_set_fft_parallel.argtypes = [C.c_int]
    return _LIB


def refpin():
    """The reference's own ThomasAlgorithm / ParaxialEquation, compiled from its
    sources (None when that library was not built)."""
    global _REFPIN
    if _REFPIN is None:
        path = os.path.join(_HERE, "_ref", "libpaxpro_refpin.so")
        if not os.path.exists(path):
            return None
        _REFPIN = C.CDLL(path)
        d = C.POINTER(C.c_double)
        _REFPIN.ref_thomas_solve.argtypes = [d, d, d, C.c_int]
        _REFPIN.ref_paraxial_equation.argtypes = [C.c_double] * 3 + [d]
        _REFPIN.ref_node_count.restype = C.c_uint
        _REFPIN.ref_node_count.argtypes = [C.c_double] * 3
        _REFPIN.ref_run2d.argtypes = [C.c_int, C.POINTER(Grid), C.POINTER(Material), C.c_int,
                                      d, C.c_int, C.c_int, d, d, C.c_int]
        _REFPIN.ref_run3d.argtypes = [C.c_int, C.POINTER(Grid), C.POINTER(Material), C.c_int,
                                      C.c_double, C.c_double, d, C.c_int, C.c_int, d, d,
                                      C.c_int]
        _REFPIN.ref_run3d_saved.argtypes = [C.c_int, C.POINTER(Grid), C.POINTER(Material),
                                            C.c_uint, C.c_uint, d, C.c_int, d,
                                            C.POINTER(C.c_uint), C.c_int]
        _REFPIN.ref_source_field.argtypes = [C.c_int, C.POINTER(Grid), C.c_int] + \
            [C.c_double] * 7 + [d]
    return _REFPIN


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def grid(xmin, xmax, dx, zmin, zmax, dz, wavenumber, ymin=None, ymax=None, dy=None):
    g = Grid()
    g.xmin, g.xmax, g.dx = xmin, xmax, dx
    g.ymin = xmin if ymin is None else ymin
    g.ymax = xmax if ymax is None else ymax
    g.dy = dx if dy is None else dy
    g.zmin, g.zmax, g.dz = zmin, zmax, dz
    g.wavenumber = wavenumber
    return g


class MaterialSpec:
    """Keeps the ctypes Material and the arrays it points into alive."""

    def __init__(self, kind=MAT_VACUUM, **kw):
        self.m = Material()
        self.m.kind = kind
        self._keep = []
        for key in ("core_half_width", "delta_clad", "beta_clad", "ramp_beta"):
            setattr(self.m, key, float(kw.get(key, 0.0)))
        self.m.ramp_points = int(kw.get("ramp_points", 0))
        self.m.n_transverse = int(kw.get("n_transverse", 0))
        sph = kw.get("spheres")
        if sph is not None and len(sph):
            arr = (Sphere * len(sph))()
            for i, s in enumerate(sph):
                arr[i] = Sphere(*[float(v) for v in s])
            self._keep.append(arr)
            self.m.spheres = C.cast(arr, C.POINTER(Sphere))
            self.m.n_spheres = len(sph)
        csg = kw.get("csg")
        if csg is not None:
            mods, parts, shapes = csg
            cm = (CsgModule * max(len(mods), 1))(*[CsgModule(*m) for m in mods])
            cp = (CsgPart * max(len(parts), 1))(*[CsgPart(*p) for p in parts])
            cs = (CsgShape * max(len(shapes), 1))(
                *[CsgShape(k, op, (C.c_double * 16)(*T), (C.c_double * 3)(*sz))
                  for k, op, T, sz in shapes])
            self._keep += [cm, cp, cs]
            self.m.csg_modules = C.cast(cm, C.c_void_p)
            self.m.csg_parts = C.cast(cp, C.c_void_p)
            self.m.csg_shapes = C.cast(cs, C.c_void_p)
            self.m.n_csg_modules = len(mods)
        if kw.get("delta_table") is not None:
            dt = np.ascontiguousarray(kw["delta_table"], dtype=np.float64)
            bt = np.ascontiguousarray(kw["beta_table"], dtype=np.float64)
            self._keep += [dt, bt]
            self.m.delta_table, self.m.beta_table = _p(dt), _p(bt)
            self.m.n_transverse = len(dt)


def node_count(mn, mx, step) -> int:
    return int(lib().orc_node_count(mn, mx, step))


def fft1d(x: np.ndarray, sign: int) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    rc = lib().orc_fft1d(_p(a), len(a), sign)
    if rc:
        raise ValueError("length must be positive")
    return a


def thomas(diag, sub, rhs) -> np.ndarray:
    d = np.ascontiguousarray(diag, dtype=np.complex128).copy()
    s = np.ascontiguousarray(sub, dtype=np.complex128).copy()
    r = np.ascontiguousarray(rhs, dtype=np.complex128).copy()
    lib().orc_thomas(_p(d), _p(s), _p(r), len(d))
    return d


def ref_thomas(diag, sub, rhs):
    rp = refpin()
    if rp is None:
        return None
    d = np.ascontiguousarray(diag, dtype=np.complex128).copy()
    s = np.ascontiguousarray(sub, dtype=np.complex128).copy()
    r = np.ascontiguousarray(rhs, dtype=np.complex128).copy()
    rp.ref_thomas_solve(_p(d), _p(s), _p(r), len(d))
    return d


def material_eval(spec: MaterialSpec, g: Grid, x, y, z):
    d = np.zeros(1)
    b = np.zeros(1)
    lib().orc_material_eval(C.byref(spec.m), C.byref(g), x, y, z, _p(d), _p(b))
    return float(d[0]), float(b[0])


def _run2d(fn, g, spec, u0, nsteps, save_every, *extra):
    u0 = np.ascontiguousarray(u0, dtype=np.complex128)
    n = len(u0)
    nsave = nsteps // save_every if save_every > 0 else 0
    saves = np.zeros((max(nsave, 1), n), dtype=np.complex128)
    out = np.zeros(n, dtype=np.complex128)
    rc = fn(C.byref(g), C.byref(spec.m), *extra, _p(u0), nsteps, save_every,
            _p(saves), _p(out))
    if rc:
        raise ValueError(f"oracle rejected the problem (rc={rc})")
    return out, saves[:nsave]


def fft2d_run(g, spec, u0, nsteps, save_every=0):
    return _run2d(lib().orc_fft2d_run, g, spec, u0, nsteps, save_every)


def cn2d_run(g, spec, u0, nsteps, save_every=0, transparent=False):
    return _run2d(lib().orc_cn2d_run, g, spec, u0, nsteps, save_every, int(transparent))


def _run3d(fn, g, spec, u0, nsteps, save_every, *extra):
    u0 = np.asfortranarray(u0, dtype=np.complex128)
    ny, nx = u0.shape
    nsave = nsteps // save_every if save_every > 0 else 0
    saves = np.zeros((max(nsave, 1), nx * ny), dtype=np.complex128)
    out = np.zeros((ny, nx), dtype=np.complex128, order="F")
    flat_in = u0.reshape(-1, order="F")
    rc = fn(C.byref(g), C.byref(spec.m), *extra, _p(flat_in), nsteps, save_every,
            _p(saves), out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc:
        raise ValueError(f"oracle rejected the problem (rc={rc})")
    return out, [s.reshape((ny, nx), order="F") for s in saves[:nsave]]


# ---- the reference's own solvers (oracle/_ref, compiled from its sources) --
REF_FFT_SOLVER_2D, REF_CRANK_NICHOLSON, REF_FFT_SOLVER_3D, REF_ADI = 1, 2, 3, 4


def ref_run2d(kind, g, spec, u0, nsteps, save_every=0, transparent=False, threads=1):
    """FFTSolver2D (kind 1) / CrankNicholson (kind 2) of the reference itself,
    driven through ParaxialSimulation and Solver::step(); (last field, saves).
    The grid's z range must hold more than nsteps steps."""
    rp = refpin()
    if rp is None:
        raise RuntimeError("reference pin library not built")
    u0 = np.ascontiguousarray(u0, dtype=np.complex128)
    n = len(u0)
    nsave = nsteps // save_every if save_every > 0 else 0
    saves = np.zeros((max(nsave, 1), n), dtype=np.complex128)
    out = np.zeros(n, dtype=np.complex128)
    rc = rp.ref_run2d(int(kind), C.byref(g), C.byref(spec.m), int(transparent), _p(u0),
                      int(nsteps), int(save_every), _p(saves), _p(out), int(threads))
    if rc:
        raise ValueError(f"reference run failed (rc={rc})")
    return out, saves[:nsave]


def ref_run3d(kind, g, spec, u0, nsteps, save_every=0, use_tbc=False, absorber_width=0.0,
              absorber_damping=0.0, threads=1):
    """FFTSolver3D (kind 3) / ADI (kind 4) of the reference itself; fields
    (Ny, Nx) Fortran-order as the oracle's 3-D runs."""
    rp = refpin()
    if rp is None:
        raise RuntimeError("reference pin library not built")
    u0 = np.asfortranarray(u0, dtype=np.complex128)
    ny, nx = u0.shape
    nsave = nsteps // save_every if save_every > 0 else 0
    saves = np.zeros((max(nsave, 1), nx * ny), dtype=np.complex128)
    out = np.zeros((ny, nx), dtype=np.complex128, order="F")
    flat_in = u0.reshape(-1, order="F")
    rc = rp.ref_run3d(int(kind), C.byref(g), C.byref(spec.m), int(use_tbc),
                      float(absorber_width), float(absorber_damping), _p(flat_in), int(nsteps),
                      int(save_every), _p(saves), out.ctypes.data_as(C.POINTER(C.c_double)),
                      int(threads))
    if rc:
        raise ValueError(f"reference run failed (rc={rc})")
    return out, [s.reshape((ny, nx), order="F") for s in saves[:nsave]]


def ref_saved_cube(kind, g, spec, u0, nsteps, ratio_x, ratio_z, threads=1):
    """The reference's saved-slice cube (Solver3D::getSolution3D) after
    nsteps steps with transverse / longitudinal downsampling ratios: a list
    of (m, m) Fortran-order slices."""
    rp = refpin()
    if rp is None:
        raise RuntimeError("reference pin library not built")
    u0 = np.asfortranarray(u0, dtype=np.complex128)
    dims = (C.c_uint * 3)()
    flat_in = u0.reshape(-1, order="F")
    rc = rp.ref_run3d_saved(int(kind), C.byref(g), C.byref(spec.m), int(ratio_x), int(ratio_z),
                            _p(flat_in), int(nsteps), None, dims, int(threads))
    if rc:
        raise ValueError(f"reference run failed (rc={rc})")
    m, _, ns = dims[0], dims[1], dims[2]
    out = np.zeros(m * m * ns, dtype=np.complex128)
    rc = rp.ref_run3d_saved(int(kind), C.byref(g), C.byref(spec.m), int(ratio_x), int(ratio_z),
                            _p(flat_in), int(nsteps), _p(out), dims, int(threads))
    if rc:
        raise ValueError(f"reference run failed (rc={rc})")
    return [out[s * m * m:(s + 1) * m * m].reshape((m, m), order="F") for s in range(ns)]


def ref_source_field(dim, g, source, wavelength, waist=1.0, cx=0.0, cy=0.0, amplitude=1.0,
                     angle_deg=0.0, z0=0.0):
    """The initial field ParaxialSimulation::setBoundaryConditions gives a
    solver: source 0 = GaussianBeam, 1 = PlaneWave; dim 2 (Nx values) or 3
    ((Ny, Nx) Fortran order)."""
    rp = refpin()
    if rp is None:
        raise RuntimeError("reference pin library not built")
    n = node_count(g.xmin, g.xmax, g.dx)
    out = np.zeros(n if dim == 2 else n * n, dtype=np.complex128)
    rc = rp.ref_source_field(int(dim), C.byref(g), int(source), float(wavelength), float(waist),
                             float(cx), float(cy), float(amplitude), float(angle_deg), float(z0),
                             _p(out))
    if rc:
        raise ValueError(f"reference source failed (rc={rc})")
    return out if dim == 2 else out.reshape((n, n), order="F")


def fft3d_run(g, spec, u0, nsteps, save_every=0, absorber_width=0.0, absorber_damping=0.0):
    return _run3d(lib().orc_fft3d_run, g, spec, u0, nsteps, save_every,
                  float(absorber_width), float(absorber_damping))


def adi3d_run(g, spec, u0, nsteps, save_every=0, use_tbc=False):
    return _run3d(lib().orc_adi3d_run, g, spec, u0, nsteps, save_every, int(use_tbc))


def gaussian_beam_2d(g, wavelength, waist, center=0.0, amplitude=1.0, z=0.0):
    n = node_count(g.xmin, g.xmax, g.dx)
    out = np.zeros(n, dtype=np.complex128)
    lib().orc_gaussian_beam_2d(C.byref(g), wavelength, waist, center, amplitude, z, _p(out))
    return out


def gaussian_beam_3d(g, wavelength, waist, cx=0.0, cy=0.0, amplitude=1.0, z=0.0):
    nx = node_count(g.xmin, g.xmax, g.dx)
    ny = node_count(g.ymin, g.ymax, g.dy)
    out = np.zeros((ny, nx), dtype=np.complex128, order="F")
    lib().orc_gaussian_beam_3d(C.byref(g), wavelength, waist, cx, cy, amplitude, z,
                               out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def block_average(field, ratio: int):
    """Saved-slice downsampling of Solver3D (src/solver3D.cpp:94-112): an
    n x n field to (n // ratio) x (n // ratio)."""
    f = np.asfortranarray(np.asarray(field, dtype=np.complex128))
    n = f.shape[0]
    m = n // int(ratio)
    out = np.zeros((m, m), dtype=np.complex128, order="F")
    lib().orc_block_average(f.ctypes.data_as(C.POINTER(C.c_double)), n, m,
                            out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def material_planes(g, spec, kind, first_step, nsteps):
    """The per-step planes the reference samples for a 3-D kind (3 =
    FFTSolver3D: the refraction material of each step; 4 = ADI: the x and y
    half-step planes), as pxp_set_material_planes takes them: (delta, beta),
    each of shape (nplanes, Nx*Ny) in the field's column-major layout."""
    n = node_count(g.xmin, g.xmax, g.dx)
    per = 2 if kind == 4 else 1
    d = np.zeros((nsteps * per, n * n))
    b = np.zeros_like(d)
    rc = lib().orc_material_planes(C.byref(g), C.byref(spec.m), int(kind), int(first_step),
                                   int(nsteps), _p(d), _p(b))
    if rc:
        raise ValueError(f"oracle rejected the planes (rc={rc})")
    return d, b


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def set_fft_parallel(on: bool) -> None:
    lib().orc_set_fft_parallel(int(bool(on)))
