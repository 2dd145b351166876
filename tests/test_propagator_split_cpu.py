"""The FFTSolver3D propagator as the product of its x and y factors.

FFTSolver3D::kernel (src/fftSolver3D.cpp:24-30) evaluates exp(-i phi) with
phi = fl(a * fl(kx^2 + ky^2)); the x pass multiplies instead by the two
factors exp(-i a kx^2) and exp(-i a ky^2), each from a table whose phase is
reduced in extended precision.  They differ by the rounding of phi (up to
about 1e-13 rad at the largest frequencies of the benchmark grids, where
phi reaches 1.3e3 rad), the same at every step.  This restates a step of
FFT propagation in FP64 (numpy's FFT, vacuum) with both forms on the
benchmark's grid spacing and wavelength, on a field with much energy at
high spatial frequencies (a strong phase object plus noise), and bounds the
drift over the steps far inside the 1e-10 parity tolerance."""
import numpy as np


def test_split_propagator_stays_within_parity_tolerance():
    n, dx = 256, 2000.0 / 4096
    k, dz = 2 * np.pi / 0.1, 2000.0
    a = 0.5 * dz / k
    idx = np.arange(n)
    kx = 2 * np.pi * np.where(idx > n // 2, n - idx, idx) / (dx * n)
    kx2 = kx * kx
    phi = a * (kx2[:, None] + kx2[None, :])
    assert phi.max() > 1.0e3
    joint = np.exp(-1j * phi)
    phase = np.longdouble(a) * kx2.astype(np.longdouble)
    fx = (np.cos(phase) - 1j * np.sin(phase)).astype(np.complex128)
    split = fx[:, None] * fx[None, :]
    rng = np.random.default_rng(0)
    x = (np.arange(n) - n / 2) * dx
    r2 = x[:, None] ** 2 + x[None, :] ** 2
    u0 = np.exp(0.5j * np.exp(-r2 / 30.0 ** 2)) * (1 + 0.01 * rng.standard_normal((n, n)))
    uj, us = u0.copy(), u0.copy()
    errs = {}
    for s in range(1, 301):
        uj = np.fft.ifft2(np.fft.fft2(uj) * joint)
        us = np.fft.ifft2(np.fft.fft2(us) * split)
        if s in (10, 100, 300):
            errs[s] = np.linalg.norm(us - uj) / np.linalg.norm(uj)
    assert errs[300] < 1e-12, errs
    # the difference grows about linearly (the same rounding every step)
    assert errs[300] > errs[10]
