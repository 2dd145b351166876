"""CPU checks of the drop-in boundary: the in-tree CUDA library loads and
exports every entry point include/paxpro_b200.h declares.  No compute calls:
this container has no GPU."""
import ctypes as C
import os

from paxpro_b200 import _capi


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_capi.LIB_PATH)
    declared = _capi.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert missing == []


def test_every_header_under_include_is_covered():
    inc = os.path.join(os.path.dirname(_capi.HEADER))
    headers = [f for f in os.listdir(inc) if f.endswith(".h")]
    assert "paxpro_b200.h" in headers


def test_node_count_matches_reference_expression():
    lib = _capi.lib()
    for mn, mx, st in [(-250.0, 250.0, 500.0 / 2047), (0.0, 4e6, 1000.0), (-1.0, 1.0, 0.3)]:
        assert lib.pxp_node_count(mn, mx, st) == int((mx - mn) / st + 1.0)


def test_status_strings():
    lib = _capi.lib()
    assert lib.pxp_status_string(0) == b"ok"
    assert b"unsupported" in lib.pxp_status_string(-7)
    assert b"sm_100a" in lib.pxp_build_info()


def test_null_arguments_are_rejected_without_a_device():
    lib = _capi.lib()
    assert lib.pxp_solver_create(None, None) == _capi.PXP_ERR_INVALID
    assert lib.pxp_step(None, 1) == _capi.PXP_ERR_INVALID
    assert lib.pxp_solver_destroy(None) == _capi.PXP_OK


def test_transverse_downsampling_of_2d_solvers_is_rejected_before_any_device_call():
    import ctypes as C
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D, x=pxp.Disc(-250.0, 250.0, 0.5, 2),
                           z=pxp.Disc(0.0, 1e4, 1000.0), wavenumber=62.8)
    h = C.c_void_p()
    rc = _capi.lib().pxp_solver_create(C.byref(spec.to_c()), C.byref(h))
    assert rc == _capi.PXP_ERR_UNSUPPORTED
    assert "downsampling" in _capi.last_error()


def test_transparent_ends_on_a_padded_cn_grid_are_rejected_before_any_device_call():
    """CrankNicholson takes any Nx with Dirichlet ends; transparent ends need
    Nx / 8 to be a power of two (the kernel pads other sizes)."""
    import ctypes as C
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi
    from paxpro_b200 import workloads as wl
    dx = wl.step_for_nodes(-250.0, 250.0, 300)
    spec = pxp.ProblemSpec(kind=pxp.CRANK_NICHOLSON, x=pxp.Disc(-250.0, 250.0, dx),
                           z=pxp.Disc(0.0, 1e4, 500.0), wavenumber=62.8, transparent_bc=True)
    h = C.c_void_p()
    rc = _capi.lib().pxp_solver_create(C.byref(spec.to_c()), C.byref(h))
    assert rc == _capi.PXP_ERR_UNSUPPORTED


def test_new_entry_points_reject_null_handles_and_fill_defaults():
    """The far-field, reference, flux and resized-post entry points reject a
    null handle without touching a device; pxp_farfield_defaults fills the
    reference's FarField defaults (angles -90..90, zero padding)."""
    import ctypes as C
    from paxpro_b200 import _capi
    lib = _capi.lib()
    p = _capi.FarFieldParams()
    p.phi_min = 3.0
    p.pad_length = 7
    lib.pxp_farfield_defaults(C.byref(p))
    assert (p.pad_length, p.phi_min, p.phi_max, p.padding) == (0, -90.0, 90.0, _capi.PAD_ZERO)
    assert (p.export_rows, p.export_cols, p.subtract_reference) == (0, 0, 0)
    out = (C.c_double * 4)()
    r, c = C.c_uint(), C.c_uint()
    assert lib.pxp_farfield(None, C.byref(p), out) == _capi.PXP_ERR_INVALID
    assert lib.pxp_farfield_shape(None, C.byref(p), C.byref(r), C.byref(c)) == _capi.PXP_ERR_INVALID
    assert lib.pxp_set_reference(None, None) == _capi.PXP_ERR_INVALID
    assert lib.pxp_set_reference_from(None, None) == _capi.PXP_ERR_INVALID
    assert lib.pxp_set_flux_windows(None, 1, 0, None, None) == _capi.PXP_ERR_INVALID
    assert lib.pxp_get_flux(None, 1, 1, out) == _capi.PXP_ERR_INVALID
    assert lib.pxp_field_flux(None, 0, 1, out) == _capi.PXP_ERR_INVALID
    assert lib.pxp_get_post_resized(None, 0, -1, 2, 2, out) == _capi.PXP_ERR_INVALID


def test_noalloc_refuses_too_many_spheres_on_a_plane_before_running_anything():
    """pxp_adi_steps_noalloc checks every plane its steps sample before the
    first launch: with 17 spheres meeting the plane of a later step the call
    is refused, having made no device call (none is possible here) and left
    the field buffer as it was."""
    import ctypes as C
    import numpy as np
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi
    from paxpro_b200 import workloads as wl
    n = 64
    dx = wl.step_for_nodes(-500.0, 500.0, n)
    spec = pxp.ProblemSpec(kind=pxp.ADI, x=pxp.Disc(-500.0, 500.0, dx),
                           y=pxp.Disc(-500.0, 500.0, dx), z=pxp.Disc(0.0, 1e4, 1000.0),
                           wavenumber=wl.K)
    # 17 spheres around z = 5000 (step 5); steps 1-4 meet none
    sph = (_capi.SphereC * 17)(*[_capi.SphereC(10.0 * i, 0.0, 5000.0, 100.0, 1e-5, 1e-7)
                                 for i in range(17)])
    field = np.arange(2 * n * n, dtype=np.float64)
    before = field.copy()
    rc = _capi.lib().pxp_adi_steps_noalloc(C.byref(spec.to_c()), sph, 17,
                                          C.c_void_p(field.ctypes.data), 1, 6, None)
    assert rc == _capi.PXP_ERR_UNSUPPORTED
    assert "nothing was run" in _capi.last_error()
    assert np.array_equal(field, before)
