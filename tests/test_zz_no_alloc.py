"""pxp_adi_steps_noalloc: ADI steps on a caller-owned device field with no
device allocation, for callers that cannot allocate device memory while they
run (memory owned by another allocator, latency-critical loops where
cudaMalloc would synchronise the device).

The test advances the same problem twice in a row through the new entry
point and through the solver-handle entry points, and requires the two to
agree within the FP64 parity tolerance (1e-10 relative L2) after each call.
Device memory for the field is allocated by the test itself (torch); the
entry point allocates nothing, so a repeat call leaves the free device memory
unchanged.  This file is collected last so that a failure here cannot hide
the other tests."""
import ctypes as C

import numpy as np
import pytest

from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _problem(pxp, n, zmin, dz, nsteps):
    L = 1000.0
    dx = wl.step_for_nodes(-L / 2, L / 2, n)
    return pxp.ProblemSpec(kind=pxp.ADI, x=pxp.Disc(-L / 2, L / 2, dx),
                           y=pxp.Disc(-L / 2, L / 2, dx),
                           z=pxp.Disc(zmin, zmin + nsteps * dz, dz), wavenumber=wl.K)


def test_noalloc_matches_solver_handle_on_two_calls():
    import torch

    import paxpro_b200 as pxp
    from paxpro_b200 import _capi

    n, dz, per_call = 256, 1000.0, 3
    spheres = [(40.0, -30.0, 2000.0, 150.0, 4.5e-5, 3.6e-6),
               (-120.0, 90.0, 5000.0, 100.0, 2e-5, 1e-6)]
    spec = _problem(pxp, n, 0.0, dz, 2 * per_call)
    rng = np.random.default_rng(11)
    u0 = (np.ones((n, n)) + 0.05 * rng.standard_normal((n, n))).astype(np.complex128)
    u0 = np.asfortranarray(u0)

    # reference: the solver-handle entry points
    ref = []
    with pxp.Solver(spec) as s:
        s.set_material_spheres([pxp.Sphere(*sp) for sp in spheres])
        s.set_initial_conditions(u0)
        for _ in range(2):
            s.step(per_call)
            ref.append(s.get_last_solution())

    # the no-allocation entry point on a field the caller owns
    lib = _capi.lib()
    prob = spec.to_c()
    arr = (_capi.SphereC * len(spheres))(*[_capi.SphereC(*sp) for sp in spheres])
    flat = torch.from_numpy(np.ascontiguousarray(u0.reshape(-1, order="F"))).to("cuda:0")
    torch.cuda.synchronize()
    got = []
    free_before_second = None
    for call in range(2):
        if call == 1:
            free_before_second = torch.cuda.mem_get_info()[0]
        rc = lib.pxp_adi_steps_noalloc(C.byref(prob), arr, len(spheres),
                                       C.c_void_p(flat.data_ptr()), 1 + call * per_call, per_call,
                                       None)
        assert rc == 0, _capi.last_error()
        torch.cuda.synchronize()
        got.append(flat.cpu().numpy().reshape((n, n), order="F").copy())
    assert torch.cuda.mem_get_info()[0] == free_before_second

    for g, r in zip(got, ref):
        assert np.linalg.norm(g - r) / np.linalg.norm(r) <= FP64_TOL
    assert np.std(np.abs(got[1])) > 1e-3  # the spheres were crossed


def test_noalloc_rejects_grids_beyond_the_scratch_limit():
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi

    spec = _problem(pxp, 1024, 0.0, 1000.0, 2)  # 1024^2 complex128 = 16 MiB > 4 MiB
    rc = _capi.lib().pxp_adi_steps_noalloc(C.byref(spec.to_c()), None, 0, C.c_void_p(1), 1, 1,
                                          None)
    assert rc == _capi.PXP_ERR_UNSUPPORTED
    assert "4 MiB" in _capi.last_error()
