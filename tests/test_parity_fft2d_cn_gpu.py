"""GPU parity of the 1-transverse-dim solvers (FFTSolver2D, CrankNicholson)
against the CPU oracle, through the C ABI.

Tolerances: FP64 plain mode <= 1e-10 relative L2 at every saved step (the
target stated for the reference path); FP32 served mode <= 1e-4 relative L2
of the intensity |u|^2 against the FP64 oracle."""
import math

import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_INT_TOL = 1e-4


def _pxp():
    import paxpro_b200 as pxp
    return pxp


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _int_rel(a, b):
    ia, ib = np.abs(a) ** 2, np.abs(b) ** 2
    return np.linalg.norm(ia - ib) / np.linalg.norm(ib)


def _oracle_2d(p, delta, beta, u0, nsteps, save_every, transparent=False):
    g = po.grid(p.xmin, p.xmax, p.dx, p.zmin, p.zmax, p.dz, wl.K)
    spec = po.MaterialSpec(po.MAT_XTABLE, delta_table=delta, beta_table=beta)
    if p.kind == "fft":
        return po.fft2d_run(g, spec, u0, nsteps, save_every)
    return po.cn2d_run(g, spec, u0, nsteps, save_every, transparent)


def _gpu_2d(p, delta, beta, u0, nsteps, save_every, precision, transparent=False, chunks=1):
    pxp = _pxp()
    kind = pxp.FFT_SOLVER_2D if p.kind == "fft" else pxp.CRANK_NICHOLSON
    spec = pxp.ProblemSpec(kind=kind, x=pxp.Disc(p.xmin, p.xmax, p.dx),
                           z=pxp.Disc(p.zmin, p.zmax, p.dz), wavenumber=wl.K,
                           precision=precision, save_every=save_every,
                           transparent_bc=transparent)
    with pxp.Solver(spec) as s:
        s.set_material_table(delta, beta)
        s.set_initial_conditions(u0)
        done = 0
        for c in range(chunks):
            k = nsteps // chunks if c < chunks - 1 else nsteps - done
            s.step(k)
            done += k
        s.synchronize()
        out = s.get_last_solution()
        saves = [s.get_saved(i) for i in range(s.num_saved())]
    return out, saves


def test_waveguide_fft2d_fp64_every_save_within_1e10():
    p = wl.waveguide_fft2d()
    d, b = p.material()
    u0 = p.initial_field()
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, p.nsteps, 100)
    out, saves = _gpu_2d(p, d, b, u0, p.nsteps, 100, 0)
    assert len(saves) == len(ref_saves) == 40
    errs = [_rel(g, r) for g, r in zip(saves, ref_saves)]
    assert max(errs) <= FP64_TOL, errs
    assert _rel(out, ref_out) <= FP64_TOL


@pytest.mark.parametrize("n", [16, 256, 1024, 4096, 8192])
def test_fft2d_fp64_sizes(n):
    p = wl.Problem2D("t", "fft", -250.0, 250.0, wl.step_for_nodes(-250.0, 250.0, n),
                     0.0, 1e6, 1000.0, 60, 15.0, wl.Waveguide())
    d, b = p.material()
    rng = np.random.default_rng(n)
    u0 = p.initial_field() + 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, 60, 20)
    out, saves = _gpu_2d(p, d, b, u0, 60, 20, 0, chunks=3)
    assert max(_rel(g, r) for g, r in zip(saves, ref_saves)) <= FP64_TOL
    assert _rel(out, ref_out) <= FP64_TOL


def test_waveguide_cn_fp64_every_save_within_1e10():
    p = wl.waveguide_cn()
    d, b = p.material()
    u0 = p.initial_field()
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, p.nsteps, 100)
    out, saves = _gpu_2d(p, d, b, u0, p.nsteps, 100, 0)
    assert len(saves) == 80
    errs = [_rel(g, r) for g, r in zip(saves, ref_saves)]
    assert max(errs) <= FP64_TOL, max(errs)


@pytest.mark.parametrize("n", [16, 64, 512, 2048])
@pytest.mark.parametrize("transparent", [False, True])
def test_cn_fp64_sizes_and_boundaries(n, transparent):
    p = wl.Problem2D("t", "cn", -250.0, 250.0, wl.step_for_nodes(-250.0, 250.0, n),
                     0.0, 1e6, 500.0, 50, 15.0, wl.Waveguide(), center=60.0)
    d, b = p.material()
    u0 = p.initial_field()
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, 50, 10, transparent)
    out, saves = _gpu_2d(p, d, b, u0, 50, 10, 0, transparent=transparent, chunks=2)
    assert max(_rel(g, r) for g, r in zip(saves, ref_saves)) <= FP64_TOL
    assert _rel(out, ref_out) <= FP64_TOL


def test_fft2d_fp32_served_intensity_within_1e4():
    p = wl.waveguide_fft2d()
    d, b = p.material()
    u0 = p.initial_field()
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, p.nsteps, 100)
    out, saves = _gpu_2d(p, d, b, u0, p.nsteps, 100, 1)
    errs = [_int_rel(g, r) for g, r in zip(saves, ref_saves)]
    assert max(errs) <= FP32_INT_TOL, max(errs)


def test_cn_fp32_served_intensity_within_1e4():
    p = wl.waveguide_cn(nsteps=2000)
    d, b = p.material()
    u0 = p.initial_field()
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, p.nsteps, 100)
    out, saves = _gpu_2d(p, d, b, u0, p.nsteps, 100, 1)
    errs = [_int_rel(g, r) for g, r in zip(saves, ref_saves)]
    assert max(errs) <= FP32_INT_TOL, max(errs)


def test_z_varying_planes_fft2d_and_cn():
    # material switched on for a band of steps, supplied as per-step planes
    for kind in ("fft", "cn"):
        n, nsteps = 512, 40
        p = wl.Problem2D("t", kind, -250.0, 250.0, wl.step_for_nodes(-250.0, 250.0, n),
                         0.0, 1e6, 500.0, nsteps, 15.0, wl.Waveguide())
        d, b = p.material()
        u0 = p.initial_field()
        # oracle with the z-invariant table for reference trajectory
        ref_out, _ = _oracle_2d(p, d, b, u0, nsteps, 0)
        pxp = _pxp()
        kd = pxp.FFT_SOLVER_2D if kind == "fft" else pxp.CRANK_NICHOLSON
        spec = pxp.ProblemSpec(kind=kd, x=pxp.Disc(p.xmin, p.xmax, p.dx),
                               z=pxp.Disc(p.zmin, p.zmax, p.dz), wavenumber=wl.K)
        per = 1 if kind == "fft" else 2
        with pxp.Solver(spec) as s:
            s.set_material_planes(np.tile(d, nsteps * per), np.tile(b, nsteps * per), 1, nsteps)
            s.set_initial_conditions(u0)
            s.step(nsteps)
            out = s.get_last_solution()
            with pytest.raises(pxp.PxpError):
                s.step(1)  # beyond the planes provided
        assert _rel(out, ref_out) <= FP64_TOL


def test_api_errors_and_counters():
    pxp = _pxp()
    p = wl.waveguide_fft2d(nsteps=10)
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D, x=pxp.Disc(p.xmin, p.xmax, p.dx),
                           z=pxp.Disc(p.zmin, p.zmax, p.dz), wavenumber=wl.K, save_every=5)
    with pxp.Solver(spec) as s:
        with pytest.raises(pxp.PxpError):
            s.step(1)  # no initial conditions yet
        s.set_initial_conditions(p.initial_field())
        assert s.current_step == 1
        s.step(10)
        assert s.current_step == 11 and s.num_saved() == 2
        with pytest.raises(pxp.PxpError):
            s.get_saved(2)
        s.reset()
        assert s.current_step == 1
    with pytest.raises(pxp.PxpError):
        # Nx = 5000 in FP64: its Bluestein length 16384 is beyond the FP64 limit
        pxp.Solver(pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D, x=pxp.Disc(0, 4999, 1.0),
                                   z=pxp.Disc(0, 10, 1.0), wavenumber=wl.K))
    with pytest.raises(pxp.PxpError):
        pxp.Solver(pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D, x=pxp.Disc(0, 4, 1.0),
                                   z=pxp.Disc(0, 10, 1.0), wavenumber=wl.K))  # Nx = 5


@pytest.mark.parametrize("n,precision", [(300, 0), (1000, 0), (2500, 0), (17, 0), (1000, 1)])
def test_cn_any_grid_size(n, precision):
    """CrankNicholson on grids whose size is not a power of two (the kernel
    pads the system with decoupled rows): every save against the oracle,
    FP64 within 1e-10, FP32 served within the intensity tolerance; the same
    with per-step material planes and with the flux windows set."""
    nsteps = 60
    p = wl.Problem2D("t", "cn", -250.0, 250.0, wl.step_for_nodes(-250.0, 250.0, n),
                     0.0, 1e6, 500.0, nsteps, 15.0, wl.Waveguide())
    d, b = p.material()
    u0 = p.initial_field()
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, nsteps, 10)
    out, saves = _gpu_2d(p, d, b, u0, nsteps, 10, precision)
    assert len(saves) == len(ref_saves)
    if precision == 0:
        assert max(_rel(g, r) for g, r in zip(saves, ref_saves)) <= FP64_TOL
        assert _rel(out, ref_out) <= FP64_TOL
    else:
        assert max(_int_rel(g, r) for g, r in zip(saves, ref_saves)) <= FP32_INT_TOL
        return
    pxp = _pxp()
    spec = pxp.ProblemSpec(kind=pxp.CRANK_NICHOLSON, x=pxp.Disc(p.xmin, p.xmax, p.dx),
                           z=pxp.Disc(p.zmin, p.zmax, p.dz), wavenumber=wl.K)
    with pxp.Solver(spec) as s:
        s.set_material_planes(np.tile(d, nsteps * 2), np.tile(b, nsteps * 2), 1, nsteps)
        s.set_initial_conditions(u0)
        s.set_flux_windows(1, np.zeros(nsteps, np.uint32), np.full(nsteps, n - 1, np.uint32))
        s.step(nsteps)
        out2 = s.get_last_solution()
        flux = s.get_flux(nsteps, 1)[0]
    assert _rel(out2, ref_out) <= FP64_TOL
    w = np.full(n, 2.0)
    w[0] = w[-1] = 1.0
    assert flux == pytest.approx(float(np.sum(w * np.abs(out2) ** 2)), rel=1e-13)


@pytest.mark.parametrize("n,precision", [(300, 0), (1000, 0), (3000, 0), (9, 0), (1000, 1)])
def test_fft2d_any_grid_size(n, precision):
    """FFTSolver2D on grids whose size is not a power of two (Bluestein's
    chirp-z transform in the kernel) against the oracle (a direct DFT for
    such lengths): FP64 within 1e-10 at every save, FP32 served within the
    intensity tolerance; per-step flux sums on the same run."""
    nsteps = 40
    p = wl.Problem2D("t", "fft", -250.0, 250.0, wl.step_for_nodes(-250.0, 250.0, n),
                     0.0, 1e6, 1000.0, nsteps, 15.0, wl.Waveguide())
    d, b = p.material()
    u0 = p.initial_field()
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, nsteps, 10)
    out, saves = _gpu_2d(p, d, b, u0, nsteps, 10, precision)
    assert len(saves) == len(ref_saves) == 4
    if precision == 1:
        assert max(_int_rel(g, r) for g, r in zip(saves, ref_saves)) <= FP32_INT_TOL
        return
    assert max(_rel(g, r) for g, r in zip(saves, ref_saves)) <= FP64_TOL
    assert _rel(out, ref_out) <= FP64_TOL
    pxp = _pxp()
    spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D, x=pxp.Disc(p.xmin, p.xmax, p.dx),
                           z=pxp.Disc(p.zmin, p.zmax, p.dz), wavenumber=wl.K)
    with pxp.Solver(spec) as s:
        s.set_material_table(d, b)
        s.set_initial_conditions(u0)
        s.set_flux_windows(1, np.zeros(nsteps, np.uint32), np.full(nsteps, n - 1, np.uint32))
        s.step(nsteps)
        out2 = s.get_last_solution()
        flux = s.get_flux(nsteps, 1)[0]
    assert _rel(out2, ref_out) <= FP64_TOL
    w = np.full(n, 2.0)
    w[0] = w[-1] = 1.0
    assert flux == pytest.approx(float(np.sum(w * np.abs(out2) ** 2)), rel=1e-13)


@pytest.mark.parametrize("planes", [False, True])
def test_fft2d_fp64_16384_two_cta_cluster(planes):
    """FFTSolver2D at 16384 points in FP64: the line (256 KB) is split by
    parity over a cluster of two CTAs that exchange halves through
    distributed shared memory; every save within 1e-10 of the oracle, with a
    z-invariant table and with per-step planes."""
    n, nsteps = 16384, 60
    p = wl.Problem2D("n16k", "fft", -500.0, 500.0, wl.step_for_nodes(-500.0, 500.0, n), 0.0,
                     1e6, 1000.0, nsteps, 20.0, wl.Waveguide())
    d, b = p.material()
    u0 = p.initial_field()
    if not planes:
        out, saves = _gpu_2d(p, d, b, u0, nsteps, 10, 0, chunks=2)
        ref_out, ref_saves = _oracle_2d(p, d, b, u0, nsteps, 10)
    else:
        pxp = _pxp()
        x = p.x
        zs = p.zmin + (np.arange(1, nsteps + 1) + 0.5) * p.dz
        dp = np.stack([np.where(np.abs(x - 1e-5 * z) <= 25.0, 0.0, 7.5e-6) for z in zs])
        bp = np.full_like(dp, 1e-7)
        spec = pxp.ProblemSpec(kind=pxp.FFT_SOLVER_2D, x=pxp.Disc(p.xmin, p.xmax, p.dx),
                               z=pxp.Disc(p.zmin, p.zmax, p.dz), wavenumber=wl.K, save_every=10)
        with pxp.Solver(spec) as s:
            s.set_material_planes(dp, bp, 1, nsteps)
            s.set_initial_conditions(u0)
            s.step(nsteps)
            out = s.get_last_solution()
            saves = [s.get_saved(i) for i in range(s.num_saved())]
        # the oracle takes the same planes one step at a time
        g = po.grid(p.xmin, p.xmax, p.dx, p.zmin, p.zmax, p.dz, wl.K)
        ref_out, ref_saves = u0, []
        for k in range(nsteps):
            gk = po.grid(p.xmin, p.xmax, p.dx, p.zmin + k * p.dz, p.zmax, p.dz, wl.K)
            spec_k = po.MaterialSpec(po.MAT_XTABLE, delta_table=dp[k], beta_table=bp[k])
            ref_out, _ = po.fft2d_run(gk, spec_k, ref_out, 1, 0)
            if (k + 1) % 10 == 0:
                ref_saves.append(ref_out)
    assert len(saves) == len(ref_saves) == nsteps // 10
    errs = [_rel(a, r) for a, r in zip(saves, ref_saves)]
    assert max(errs) <= FP64_TOL, errs
    assert _rel(out, ref_out) <= FP64_TOL


@pytest.mark.parametrize("n,precision", [(8192, 0), (16384, 0), (16384, 1), (6000, 0)])
def test_cn_cluster_sizes(n, precision):
    """CrankNicholson beyond one SM's shared memory (8192 and 16384 rows,
    and 6000 padded to 8192): the step-invariant path on a cluster of 2 or 4
    CTAs, the stencil halo and the recurrences' carries crossing CTAs
    through distributed shared memory.  FP64 within 1e-10 of the oracle at
    every save, FP32 intensity within 1e-4."""
    nsteps = 40
    p = wl.Problem2D("cn_big", "cn", -500.0, 500.0, wl.step_for_nodes(-500.0, 500.0, n), 0.0,
                     1e6, 500.0, nsteps, 20.0, wl.Waveguide())
    d, b = p.material()
    u0 = p.initial_field()
    out, saves = _gpu_2d(p, d, b, u0, nsteps, 10, precision, chunks=2)
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, nsteps, 10)
    assert len(saves) == len(ref_saves) == nsteps // 10
    if precision == 0:
        errs = [_rel(a, r) for a, r in zip(saves, ref_saves)]
        assert max(errs) <= FP64_TOL, errs
    else:
        assert max(_int_rel(a, r) for a, r in zip(saves, ref_saves)) <= FP32_INT_TOL


def test_cn_cluster_size_rejects_planes_and_transparent_ends():
    import paxpro_b200 as pxp
    from paxpro_b200 import _capi
    n = 8192
    dx = wl.step_for_nodes(-500.0, 500.0, n)
    spec = pxp.ProblemSpec(kind=pxp.CRANK_NICHOLSON, x=pxp.Disc(-500.0, 500.0, dx),
                           z=pxp.Disc(0.0, 1e4, 500.0), wavenumber=wl.K)
    with pxp.Solver(spec) as s:
        d = np.zeros((2 * 3, n))
        s.set_material_planes(d, d, 1, 3)  # z-varying: the general kernel would be needed
        s.set_initial_conditions(np.ones(n, dtype=np.complex128))
        assert _capi.lib().pxp_step(s._h, 1) == _capi.PXP_ERR_UNSUPPORTED


@pytest.mark.parametrize("n", [512, 1024, 2048, 4096])
@pytest.mark.parametrize("variant", ["0", "1"])
@pytest.mark.parametrize("precision", [0, 1])
def test_fft2d_kernel_variants(n, variant, precision, monkeypatch):
    """Both FFTSolver2D kernels the tuner chooses between at 512..4096
    points -- the shared-memory Stockham kernel (PXP_FFT1D_R16=0) and the
    register-resident radix-16 kernel (=1) -- with saves and chunked calls:
    FP64 within 1e-10 of the oracle at every save, FP32
    intensity within 1e-4 (over 600 steps)."""
    monkeypatch.setenv("PXP_FFT1D_R16", variant)
    nsteps = 60 if precision == 0 else 600
    p = wl.Problem2D("t", "fft", -250.0, 250.0, wl.step_for_nodes(-250.0, 250.0, n),
                     0.0, 1e6, 1000.0, nsteps, 15.0, wl.Waveguide())
    d, b = p.material()
    rng = np.random.default_rng(n)
    u0 = p.initial_field() + 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, nsteps, nsteps // 3)
    out, saves = _gpu_2d(p, d, b, u0, nsteps, nsteps // 3, precision, chunks=3)
    assert len(saves) == len(ref_saves) == 3
    if precision == 0:
        assert max(_rel(g, r) for g, r in zip(saves, ref_saves)) <= FP64_TOL
        assert _rel(out, ref_out) <= FP64_TOL
    else:
        assert max(_int_rel(g, r) for g, r in zip(saves, ref_saves)) <= FP32_INT_TOL


@pytest.mark.parametrize("variant", ["0", "1"])
@pytest.mark.parametrize("precision", [0, 1])
def test_cn_4096_kernel_variants(variant, precision, monkeypatch):
    """Both launches of CrankNicholson's step-invariant path at 4096 rows
    the tuner chooses between: one CTA (PXP_CN_CLUSTER=0) and a cluster of
    two CTAs exchanging the halo and the recurrences' carries through
    distributed shared memory (=1); every save against the oracle."""
    monkeypatch.setenv("PXP_CN_CLUSTER", variant)
    nsteps = 200
    p = wl.Problem2D("cn4096", "cn", -250.0, 250.0, wl.step_for_nodes(-250.0, 250.0, 4096), 0.0,
                     1e6, 500.0, nsteps, 15.0, wl.Waveguide())
    d, b = p.material()
    u0 = p.initial_field()
    out, saves = _gpu_2d(p, d, b, u0, nsteps, 50, precision, chunks=2)
    ref_out, ref_saves = _oracle_2d(p, d, b, u0, nsteps, 50)
    assert len(saves) == len(ref_saves) == 4
    if precision == 0:
        assert max(_rel(a, r) for a, r in zip(saves, ref_saves)) <= FP64_TOL
        assert _rel(out, ref_out) <= FP64_TOL
    else:
        assert max(_int_rel(a, r) for a, r in zip(saves, ref_saves)) <= FP32_INT_TOL
