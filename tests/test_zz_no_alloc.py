"""pxp_adi_steps_noalloc: ADI steps on a caller-owned device field with no
device allocation, for callers that cannot allocate device memory while they
run (memory owned by another allocator, latency-critical loops where
cudaMalloc would synchronise the device).

Each case advances the same problem twice in a row through the new entry
point and through the solver-handle entry points and requires, after each
call, agreement with the handle path and with the CPU oracle: within the FP64
parity tolerance (1e-10 relative L2) in FP64, and within the served-mode
intensity tolerance (1e-4 relative L2 of |u|^2) in FP32.  Device memory for
the field is allocated by the test itself (torch); the entry point allocates
nothing, so a repeat call leaves the free device memory unchanged.  This file
is collected last so that a failure here cannot hide the other tests."""
import ctypes as C

import numpy as np
import pytest

from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_INTENSITY_TOL = 1e-4

SPHERES = [(40.0, -30.0, 2000.0, 150.0, 4.5e-5, 3.6e-6),
           (-120.0, 90.0, 5000.0, 100.0, 2e-5, 1e-6)]


def _problem(pxp, n, dz, nsteps, precision, tbc):
    L = 1000.0
    dx = wl.step_for_nodes(-L / 2, L / 2, n)
    return pxp.ProblemSpec(kind=pxp.ADI, x=pxp.Disc(-L / 2, L / 2, dx),
                           y=pxp.Disc(-L / 2, L / 2, dx), z=pxp.Disc(0.0, nsteps * dz, dz),
                           wavenumber=wl.K, precision=precision, transparent_bc=tbc)


def _oracle(spec, u0, nsteps):
    from oracle import pyoracle as po
    g = po.grid(spec.x.min, spec.x.max, spec.x.step, spec.z.min, spec.z.max, spec.z.step, wl.K)
    out, _ = po.adi3d_run(g, po.MaterialSpec(po.MAT_SPHERES, spheres=SPHERES), u0, nsteps,
                          use_tbc=bool(spec.transparent_bc))
    return out


def _close(got, want, precision):
    if precision == 0:
        return np.linalg.norm(got - want) / np.linalg.norm(want) <= FP64_TOL
    ig, iw = np.abs(got) ** 2, np.abs(want) ** 2
    return np.linalg.norm(ig - iw) / np.linalg.norm(iw) <= FP32_INTENSITY_TOL


@pytest.mark.parametrize("n,precision,tbc,own_stream", [
    (256, 0, False, False),   # FP64, Dirichlet ends, default stream
    (256, 0, True, True),     # FP64, transparent ends, a caller stream
    (256, 1, False, True),    # FP32 (complex64 field)
    (200, 1, True, False),    # FP32, a size other than a power of two, transparent ends
    (512, 0, False, False),   # FP64 at the scratch limit: 512^2 x 16 B = 4 MiB
])
def test_noalloc_matches_solver_handle_and_oracle_on_two_calls(n, precision, tbc, own_stream):
    import torch

    import paxpro_b200 as pxp
    from paxpro_b200 import _capi

    dz, per_call = 1000.0, 3
    spec = _problem(pxp, n, dz, 2 * per_call, precision, tbc)
    rng = np.random.default_rng(11)
    u0 = np.asfortranarray((np.ones((n, n)) + 0.05 * rng.standard_normal((n, n)))
                           .astype(np.complex128))
    if precision == 1:  # both paths start from the same complex64 values
        u0 = np.asfortranarray(u0.astype(np.complex64).astype(np.complex128))

    handle = []
    with pxp.Solver(spec) as s:
        s.set_material_spheres([pxp.Sphere(*sp) for sp in SPHERES])
        s.set_initial_conditions(u0)
        for _ in range(2):
            s.step(per_call)
            handle.append(s.get_last_solution())
    oracle = [_oracle(spec, u0, per_call), _oracle(spec, u0, 2 * per_call)]

    lib = _capi.lib()
    prob = spec.to_c()
    arr = (_capi.SphereC * len(SPHERES))(*[_capi.SphereC(*sp) for sp in SPHERES])
    dt = torch.complex128 if precision == 0 else torch.complex64
    flat = torch.from_numpy(np.ascontiguousarray(u0.reshape(-1, order="F"))).to(dt).to("cuda:0")
    stream = torch.cuda.Stream() if own_stream else None
    torch.cuda.synchronize()
    got = []
    free_before_second = None
    for call in range(2):
        if call == 1:
            free_before_second = torch.cuda.mem_get_info()[0]
        rc = lib.pxp_adi_steps_noalloc(C.byref(prob), arr, len(SPHERES),
                                       C.c_void_p(flat.data_ptr()), 1 + call * per_call, per_call,
                                       C.c_void_p(stream.cuda_stream) if stream else None)
        assert rc == 0, _capi.last_error()
        torch.cuda.synchronize()
        got.append(flat.cpu().numpy().astype(np.complex128).reshape((n, n), order="F").copy())
    assert torch.cuda.mem_get_info()[0] == free_before_second

    for g, h, o in zip(got, handle, oracle):
        assert _close(g, h, precision)
        assert _close(g, o, precision)
    assert np.std(np.abs(got[1])) > 1e-3  # the spheres were crossed


def test_noalloc_rejects_grids_beyond_the_scratch_limit():
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi

    spec = _problem(pxp, 1024, 1000.0, 2, 0, False)  # 1024^2 complex128 = 16 MiB > 4 MiB
    rc = _capi.lib().pxp_adi_steps_noalloc(C.byref(spec.to_c()), None, 0, C.c_void_p(1), 1, 1,
                                          None)
    assert rc == _capi.PXP_ERR_UNSUPPORTED
    assert "4 MiB" in _capi.last_error()


def test_noalloc_keeps_the_callers_current_device():
    import torch

    import paxpro_b200 as pxp
    from paxpro_b200 import _capi

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    n = 128
    spec = _problem(pxp, n, 1000.0, 2, 0, False)
    spec.device = 1
    flat = torch.ones(n * n, dtype=torch.complex128, device="cuda:1")
    torch.cuda.set_device(0)
    rc = _capi.lib().pxp_adi_steps_noalloc(C.byref(spec.to_c()), None, 0,
                                          C.c_void_p(flat.data_ptr()), 1, 2, None)
    assert rc == 0, _capi.last_error()
    assert torch.cuda.current_device() == 0
    torch.cuda.synchronize(1)
    assert torch.isfinite(torch.view_as_real(flat)).all()
