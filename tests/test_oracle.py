"""CPU tests of the oracle: FFT against numpy, the tridiagonal solve against
the reference's own ThomasAlgorithm compiled from its source, and
known-answer tests taken from the reference's formulas."""
import math

import numpy as np
import pytest

from oracle import pyoracle as po
from paxpro_b200 import workloads as wl

LAM = 0.1
K = 2 * math.pi / LAM


@pytest.mark.parametrize("n", [8, 64, 512, 2048, 4096])
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft_matches_numpy(n, sign):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
    got = po.fft1d(x, sign)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-14


def test_fft_rejects_empty_input():
    with pytest.raises(ValueError):
        po.fft1d(np.ones(0, dtype=complex), -1)


def _random_system(n, dominance, seed):
    rng = np.random.default_rng(seed)
    sub = rng.standard_normal(n - 1) + 1j * rng.standard_normal(n - 1)
    diag = (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    mag = np.abs(np.concatenate([[0], sub])) + np.abs(np.concatenate([sub, [0]]))
    diag = diag / np.abs(diag) * mag * dominance + 1e-3
    rhs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return diag, sub, rhs


@pytest.mark.parametrize("n", [2, 3, 17, 256, 4096])
@pytest.mark.parametrize("dominance", [1.0, 1.5, 4.0])
def test_thomas_bit_exact_against_reference_source(n, dominance):
    if po.refpin() is None:
        pytest.skip("reference pin library not built (reference tree absent when building)")
    d, s, r = _random_system(n, dominance, seed=n)
    ours = po.thomas(d, s, r)
    theirs = po.ref_thomas(d, s, r)
    assert np.array_equal(ours.view(np.uint64), theirs.view(np.uint64))


@pytest.mark.parametrize("n", [4, 100, 512])
def test_thomas_matches_dense_solve(n):
    d, s, r = _random_system(n, 2.0, seed=7 * n)
    A = np.diag(d) + np.diag(s, 1) + np.diag(s, -1)
    x = po.thomas(d, s, r)
    ref = np.linalg.solve(A, r)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-12


def test_cn_matrix_thomas_on_config_ratio():
    # weakly dominant CN matrix of config 1 (rho ~ 534)
    p = wl.waveguide_cn()
    rho = p.dz / (K * p.dx * p.dx)
    assert 500 < rho < 600
    n = 512
    diag = np.full(n, 1.0 + 0.5j * rho)
    sub = np.full(n - 1, -0.25j * rho)
    rhs = np.random.default_rng(1).standard_normal(n) + 0j
    A = np.diag(diag) + np.diag(sub, 1) + np.diag(sub, -1)
    x = po.thomas(diag, sub, rhs)
    assert np.linalg.norm(A @ x - rhs) / np.linalg.norm(rhs) < 1e-12


def test_paraxial_equation_defaults_match_reference_source():
    rp = po.refpin()
    if rp is None:
        pytest.skip("reference pin library not built")
    import ctypes as C
    out = np.zeros(6)
    rp.ref_paraxial_equation(1.5, 2.5, K, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert list(out[:4]) == [1.0, 1.0, 1.0, 0.0]
    ph = np.exp(1j * K * 2.5)
    assert abs(out[4] - ph.real) < 1e-15 and abs(out[5] - ph.imag) < 1e-15


def test_node_count_truncation_and_step_choice():
    assert po.node_count(-250.0, 250.0, 500.0 / 2047) in (2047, 2048)
    step = wl.step_for_nodes(-250.0, 250.0, 2048)
    assert po.node_count(-250.0, 250.0, step) == 2048
    assert wl.node_count(-250.0, 250.0, step) == 2048


def test_waveguide_table_equals_oracle_material():
    p = wl.waveguide_fft2d()
    g = po.grid(p.xmin, p.xmax, p.dx, p.zmin, p.zmax, p.dz, K)
    d, b = p.material()
    spec = po.MaterialSpec(po.MAT_WAVEGUIDE, core_half_width=25.0, delta_clad=7.5e-6,
                           beta_clad=1e-7, ramp_points=25, ramp_beta=1e-4, n_transverse=p.nx)
    for i in list(range(0, 40)) + list(range(990, 1060)) + list(range(p.nx - 40, p.nx)):
        od, ob = po.material_eval(spec, g, p.x[i], 0.0, 0.0)
        assert od == d[i] and ob == b[i], i


def _grid3(n=128, L=2000.0, dz=1000.0, zmax=1e5):
    dx = L / (n - 1)
    return po.grid(-L / 2, L / 2, dx, 0.0, zmax, dz, K), dx


def test_k1_vacuum_fft3d_gaussian_matches_closed_form():
    g, dx = _grid3(n=256)
    w0, nsteps, dz = 100.0, 100, 1000.0
    u0 = po.gaussian_beam_3d(g, LAM, w0)
    out, _ = po.fft3d_run(g, po.MaterialSpec(), u0, nsteps)
    xs = g.xmin + np.arange(256) * dx
    X, Y = np.meshgrid(xs, xs)
    z = nsteps * dz
    zr = math.pi * w0 ** 2 / LAM
    w = w0 * math.sqrt(1 + (z / zr) ** 2)
    inv_r = z / (z * z + zr * zr)
    exact = (w0 / w) * np.exp(-(X ** 2 + Y ** 2) / w ** 2) * \
        np.exp(0.5j * K * (X ** 2 + Y ** 2) * inv_r - 1j * math.atan(z / zr))
    assert np.linalg.norm(out - exact) / np.linalg.norm(exact) < 1e-12
    # The reference's GaussianBeam::get(x, y, z) (src/gaussianBeam.cpp:57-63)
    # omits the y^2 curvature phase, so at z > 0 it is not the exact solution.
    ref_formula = po.gaussian_beam_3d(g, LAM, w0, z=z)
    assert np.linalg.norm(ref_formula - exact) / np.linalg.norm(exact) > 1e-3


def test_k5_fft2d_gaussian_one_transverse_dim_closed_form():
    n, L, w0, nsteps, dz = 1024, 2000.0, 60.0, 50, 1000.0
    dx = L / (n - 1)
    g = po.grid(-L / 2, L / 2, dx, 0.0, 1e5, dz, K)
    u0 = po.gaussian_beam_2d(g, LAM, w0)
    out, _ = po.fft2d_run(g, po.MaterialSpec(), u0, nsteps)
    xs = g.xmin + np.arange(n) * dx
    z = nsteps * dz
    zr = math.pi * w0 ** 2 / LAM
    w = w0 * math.sqrt(1 + (z / zr) ** 2)
    inv_r = z / (z * z + zr * zr)
    exact = math.sqrt(w0 / w) * np.exp(-xs ** 2 / w ** 2) * \
        np.exp(0.5j * K * xs ** 2 * inv_r - 0.5j * math.atan(z / zr))
    assert np.linalg.norm(out - exact) / np.linalg.norm(exact) < 1e-12


def test_k2_plane_wave_uniform_medium():
    n, nsteps, dz, delta, beta = 64, 40, 500.0, 3e-6, 2e-8
    g = po.grid(-100.0, 100.0, 200.0 / (n - 1), 0.0, 1e5, dz, K)
    spec = po.MaterialSpec(po.MAT_XTABLE, delta_table=np.full(n, delta),
                           beta_table=np.full(n, beta))
    out, _ = po.fft2d_run(g, spec, np.ones(n, dtype=complex), nsteps)
    t = np.exp(-K * (beta + 1j * delta) * dz)
    assert np.max(np.abs(out - t ** nsteps)) < 1e-12
    g3 = po.grid(-100.0, 100.0, 200.0 / (n - 1), 0.0, 1e5, dz, K)
    sph = po.MaterialSpec(po.MAT_SPHERES, spheres=[(0, 0, 0, 1e9, delta, beta)])
    out3, _ = po.fft3d_run(g3, sph, np.ones((n, n), dtype=complex, order="F"), nsteps)
    assert np.max(np.abs(out3 - t ** nsteps)) < 1e-12


def test_k3_unitarity_fft_vacuum_and_cn():
    rng = np.random.default_rng(3)
    n = 512
    g = po.grid(-250.0, 250.0, 500.0 / (n - 1), 0.0, 1e6, 1000.0, K)
    u0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    out, _ = po.fft2d_run(g, po.MaterialSpec(), u0, 200)
    assert abs(np.linalg.norm(out) / np.linalg.norm(u0) - 1) < 1e-13
    # Crank-Nicolson with beta = 0 and Dirichlet ends is a Cayley transform.
    spec = po.MaterialSpec(po.MAT_XTABLE, delta_table=np.full(n, 2e-6), beta_table=np.zeros(n))
    out_cn, _ = po.cn2d_run(g, spec, u0, 200)
    assert abs(np.linalg.norm(out_cn) / np.linalg.norm(u0) - 1) < 1e-11


def test_adi_vacuum_plane_wave_interior_stays_flat():
    n = 64
    g = po.grid(-500.0, 500.0, 1000.0 / (n - 1), 0.0, 1e5, 1000.0, K)
    u0 = np.ones((n, n), dtype=complex, order="F")
    out, _ = po.adi3d_run(g, po.MaterialSpec(), u0, 3)
    # Dirichlet edges disturb the border; the centre of a plane wave moves by
    # at most the boundary wave that reached it after three steps.
    c = out[n // 2 - 2:n // 2 + 2, n // 2 - 2:n // 2 + 2]
    assert np.max(np.abs(np.abs(c) - 1.0)) < 0.05


@pytest.mark.parametrize("n", [17, 300, 1000])
def test_oracle_dft_of_other_lengths_matches_numpy(n):
    """The oracle's transform of a length that is not a power of two (a
    direct DFT with exactly indexed factors) against numpy's FFT, both
    signs (unnormalised, the FFTW convention)."""
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign, want in ((-1, np.fft.fft(x)), (1, np.fft.ifft(x) * n)):
        got = po.fft1d(x, sign)
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-14
