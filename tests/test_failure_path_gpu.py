"""The failure path of the kernels' bounded waits, without a GPU fault.

The propagation kernels wait for their asynchronous copies (the ADI vacuum
kernel's table copy on an mbarrier) with a bounded wait: when it runs out,
the kernel counts it in a device counter and returns instead of hanging,
and the host reports PXP_ERR_CUDA at the next synchronisation of every
handle that existed when it happened.  pxp_selftest_bounded_wait launches a
one-thread kernel whose mbarrier expects a copy that is never issued (a flag
that nothing sets), with a 1 ms limit: the wait runs out, nothing faults, the
handle reports the error, and the context stays usable for new handles."""
import ctypes as C

import numpy as np
import pytest

from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _adi_spec(pxp, n=64):
    dx = wl.step_for_nodes(-500.0, 500.0, n)
    return pxp.ProblemSpec(kind=pxp.ADI, x=pxp.Disc(-500.0, 500.0, dx),
                           y=pxp.Disc(-500.0, 500.0, dx), z=pxp.Disc(0.0, 1e4, 1000.0),
                           wavenumber=wl.K)


def test_bounded_wait_runs_out_and_is_reported():
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi
    lib = _capi.lib()
    n = 64
    u0 = np.ones((n, n), dtype=np.complex128, order="F")
    with pxp.Solver(_adi_spec(pxp, n)) as s:
        s.set_initial_conditions(u0)
        s.step(2)
        assert lib.pxp_synchronize(s._h) == _capi.PXP_OK
        assert lib.pxp_selftest_bounded_wait(s._h, 1_000_000) == _capi.PXP_OK  # 1 ms
        rc = lib.pxp_synchronize(s._h)
        assert rc == _capi.PXP_ERR_CUDA
        assert "bounded wait" in _capi.last_error(s._h)
    # the context is still usable: a new handle steps and reads back normally
    with pxp.Solver(_adi_spec(pxp, n)) as s2:
        s2.set_initial_conditions(u0)
        s2.step(3)
        assert lib.pxp_synchronize(s2._h) == _capi.PXP_OK
        out = s2.get_last_solution()
        assert np.all(np.isfinite(out))


def test_bounded_wait_selftest_rejects_bad_limits():
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi
    lib = _capi.lib()
    assert lib.pxp_selftest_bounded_wait(None, 1000) == _capi.PXP_ERR_INVALID
    with pxp.Solver(_adi_spec(pxp)) as s:
        assert lib.pxp_selftest_bounded_wait(s._h, 0) == _capi.PXP_ERR_INVALID
        assert lib.pxp_selftest_bounded_wait(s._h, 20_000_000_000) == _capi.PXP_ERR_INVALID
