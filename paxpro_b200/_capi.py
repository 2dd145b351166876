"""ctypes binding of the C ABI declared in include/paxpro_b200.h.

This is the Python counterpart of the reference's SWIG module
(pypaxpro/pypaxpro.i): it binds the plain-C entry points one to one.  The
library is the in-tree build paxpro_b200/lib/libpaxpro_b200.so; if it is
missing the import fails loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libpaxpro_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "paxpro_b200.h")

PXP_OK = 0
PXP_ERR_INVALID = -1
PXP_ERR_NOMEM = -2
PXP_ERR_CUDA = -3
PXP_ERR_ABORTED = -4
PXP_ERR_BUDGET = -5
PXP_ERR_NOT_READY = -6
PXP_ERR_UNSUPPORTED = -7
POST_ABS, POST_ARG, POST_REAL, POST_ABS2 = 0, 1, 2, 3

FFT_SOLVER_2D, CRANK_NICHOLSON, FFT_SOLVER_3D, ADI = 1, 2, 3, 4
FP64, FP32 = 0, 1


class Discretization(C.Structure):
    _fields_ = [("min", C.c_double), ("max", C.c_double), ("step", C.c_double),
                ("downsampling_ratio", C.c_uint)]


class Problem(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("precision", C.c_int),
        ("x", Discretization), ("y", Discretization), ("z", Discretization),
        ("wavenumber", C.c_double), ("transparent_bc", C.c_int),
        ("absorber_width", C.c_double), ("absorber_damping", C.c_double),
        ("save_every", C.c_int), ("device", C.c_int),
    ]


class SphereC(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("cx", "cy", "cz", "radius", "delta", "beta")]


class CsgShapeC(C.Structure):
    _fields_ = [("kind", C.c_int), ("operation", C.c_int), ("transform", C.c_double * 16),
                ("size", C.c_double * 3)]


class CsgPartC(C.Structure):
    _fields_ = [("operation", C.c_int), ("first_shape", C.c_int), ("num_shapes", C.c_int),
                ("delta", C.c_double), ("beta", C.c_double)]


class CsgModuleC(C.Structure):
    _fields_ = [("first_part", C.c_int), ("num_parts", C.c_int)]


PAD_ZERO, PAD_LINEAR_FIT, PAD_CONSTANT = 0, 1, 2


class FarFieldParams(C.Structure):
    _fields_ = [("pad_length", C.c_uint), ("phi_min", C.c_double), ("phi_max", C.c_double),
                ("padding", C.c_int), ("pad_value_re", C.c_double), ("pad_value_im", C.c_double),
                ("export_rows", C.c_uint), ("export_cols", C.c_uint),
                ("subtract_reference", C.c_int)]


class PxpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


_lib = None


def declared_symbols() -> list[str]:
    """Function names declared in include/paxpro_b200.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(pxp_[a-z0-9_]+)\s*\(", text)))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python paxpro_b200/build.py`")
    L = C.CDLL(LIB_PATH)
    d = C.POINTER(C.c_double)
    h = C.c_void_p
    sig = {
        "pxp_node_count": (C.c_uint, [C.c_double] * 3),
        "pxp_solver_create": (C.c_int, [C.POINTER(Problem), C.POINTER(h)]),
        "pxp_solver_destroy": (C.c_int, [h]),
        "pxp_set_material_table": (C.c_int, [h, d, d, C.c_size_t]),
        "pxp_set_material_planes": (C.c_int, [h, d, d, C.c_int, C.c_int]),
        "pxp_set_material_spheres": (C.c_int, [h, C.POINTER(SphereC), C.c_int]),
        "pxp_set_initial_conditions": (C.c_int, [h, d]),
        "pxp_set_initial_conditions_device": (C.c_int, [h, C.c_void_p]),
        "pxp_step": (C.c_int, [h, C.c_int]),
        "pxp_solve": (C.c_int, [h]),
        "pxp_synchronize": (C.c_int, [h]),
        "pxp_get_last_solution": (C.c_int, [h, d]),
        "pxp_get_field_device": (C.c_int, [h, C.POINTER(C.c_void_p), C.POINTER(C.c_int)]),
        "pxp_get_stream": (C.c_int, [h, C.POINTER(C.c_void_p)]),
        "pxp_num_saved": (C.c_int, [h, C.POINTER(C.c_int)]),
        "pxp_get_saved": (C.c_int, [h, C.c_int, d]),
        "pxp_get_post": (C.c_int, [h, C.c_int, C.c_int, d]),
        "pxp_get_post_resized": (C.c_int, [h, C.c_int, C.c_int, C.c_uint, C.c_uint, d]),
        "pxp_set_material_csg": (C.c_int, [h, C.POINTER(CsgModuleC), C.c_int, C.POINTER(CsgPartC),
                                           C.c_int, C.POINTER(CsgShapeC), C.c_int]),
        "pxp_saved_max_abs": (C.c_int, [h, d]),
        "pxp_farfield_defaults": (None, [C.POINTER(FarFieldParams)]),
        "pxp_farfield_shape": (C.c_int, [h, C.POINTER(FarFieldParams), C.POINTER(C.c_uint),
                                         C.POINTER(C.c_uint)]),
        "pxp_farfield": (C.c_int, [h, C.POINTER(FarFieldParams), d]),
        "pxp_set_reference": (C.c_int, [h, d]),
        "pxp_set_reference_from": (C.c_int, [h, h]),
        "pxp_set_flux_windows": (C.c_int, [h, C.c_int, C.c_int, C.POINTER(C.c_uint),
                                           C.POINTER(C.c_uint)]),
        "pxp_get_flux": (C.c_int, [h, C.c_int, C.c_int, d]),
        "pxp_field_flux": (C.c_int, [h, C.c_uint, C.c_uint, d]),
        "pxp_reset": (C.c_int, [h]),
        "pxp_current_step": (C.c_int, [h, C.POINTER(C.c_uint)]),
        "pxp_shape": (C.c_int, [h, C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.POINTER(C.c_uint)]),
        "pxp_selftest_bounded_wait": (C.c_int, [h, C.c_ulonglong]),
        "pxp_adi_steps_noalloc": (C.c_int, [C.POINTER(Problem), C.POINTER(SphereC), C.c_int,
                                            C.c_void_p, C.c_uint, C.c_int, C.c_void_p]),
        "pxp_device_bytes": (C.c_int, [h, C.POINTER(C.c_size_t)]),
        "pxp_get_intensity": (C.c_int, [h, d]),
        "pxp_batch_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(h)]),
        "pxp_batch_destroy": (C.c_int, [h]),
        "pxp_batch_admit": (C.c_int, [h, h, C.c_int]),
        "pxp_batch_round": (C.c_int, [h, C.c_int]),
        "pxp_batch_collect": (C.c_int, [h, C.POINTER(h), C.c_int, C.POINTER(C.c_int)]),
        "pxp_batch_status": (C.c_int, [h, C.POINTER(C.c_int), C.POINTER(C.c_size_t)]),
        "pxp_last_error": (C.c_int, [h, C.c_char_p, C.c_size_t]),
        "pxp_status_string": (C.c_char_p, [C.c_int]),
        "pxp_build_info": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error(handle=None) -> str:
    buf = C.create_string_buffer(1024)
    lib().pxp_last_error(handle, buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, handle=None) -> None:
    if status != PXP_OK:
        raise PxpError(status, last_error(handle) or lib().pxp_status_string(status).decode())
