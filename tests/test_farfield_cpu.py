"""The far-field oracle (oracle/farfield.py, post::FarField restated) against
closed forms: the padded transform of a constant line is a Dirichlet kernel,
a separable 3-D field gives the product of its axis spectra with the x axis
mirrored (the conjugated rows of src/farFieldPost.cpp:227), the angle-to-index
map of :78-101 at hand-computed points, and resizeMatrix
(src/postProcessing.cpp:29-49) on a small matrix."""
import math

import numpy as np
import pytest

from oracle import farfield as ff


def test_angle_to_index_known_values():
    k, step, size = 2.0 * math.pi / 0.1, 0.5, 1000   # size*k*step/(2 pi) = 5000
    assert ff.angle_to_index(0.0, size, k, step) == 500
    assert ff.angle_to_index(0.05, size, k, step) == 500 + int(5000 * math.sin(0.05 * ff.PI / 180))
    assert ff.angle_to_index(-0.05, size, k, step) == 500 + int(-5000 * math.sin(0.05 * ff.PI / 180))
    assert ff.angle_to_index(10.0, size, k, step) == size - 1
    assert ff.angle_to_index(-10.0, size, k, step) == 0


def test_fftshift_odd_length_keeps_last_entry():
    a = np.arange(7.0)
    assert list(ff.fftshift(a)) == [3.0, 4.0, 5.0, 0.0, 1.0, 2.0, 6.0]
    assert list(ff.fftshift(np.arange(6.0))) == [3.0, 4.0, 5.0, 0.0, 1.0, 2.0]


@pytest.mark.parametrize("n,L", [(64, 512), (100, 1000), (37, 37)])
def test_2d_constant_line_is_a_dirichlet_kernel(n, L):
    k, dx = 2.0 * math.pi / 0.1, 0.05                     # L*k*dx/(2 pi) = L/2: every angle kept
    got = ff.farfield_2d(np.ones(n, dtype=np.complex128), L, -90.0, 90.0, k, dx)
    Lp = max(L, n)
    kk = np.arange(Lp)
    with np.errstate(invalid="ignore", divide="ignore"):
        d = np.abs(np.sin(np.pi * kk * n / Lp) / np.sin(np.pi * kk / Lp))
    d[0] = n
    want = ff.fftshift(d / math.sqrt(Lp))
    lo = ff.angle_to_index(-90.0, Lp, k, dx)
    assert np.allclose(got, want[lo:lo + got.shape[0]], rtol=1e-12, atol=1e-12)


def test_2d_pad_value_enters_only_the_zero_frequency():
    rng = np.random.default_rng(2)
    u = rng.standard_normal(50) + 1j * rng.standard_normal(50)
    k, dx, L, p = 2.0 * math.pi / 0.1, 0.05, 256, 0.3 - 0.2j
    a = ff.farfield_2d(u, L, -90.0, 90.0, k, dx, pad_value=p)
    b = ff.farfield_2d(u - p, L, -90.0, 90.0, k, dx)
    centre = L // 2 - ff.angle_to_index(-90.0, L, k, dx)
    mask = np.ones(a.shape[0], bool)
    mask[centre] = False
    assert np.allclose(a[mask], b[mask], rtol=1e-12, atol=1e-12)
    assert a[centre] == pytest.approx(abs(p * L + np.sum(u - p)) / math.sqrt(L), rel=1e-12)


def test_3d_separable_field_mirrors_x():
    rng = np.random.default_rng(5)
    ny = nx = 24
    ay = rng.standard_normal(ny) + 1j * rng.standard_normal(ny)
    bx = rng.standard_normal(nx) + 1j * rng.standard_normal(nx)
    u = np.outer(ay, bx)
    k, step, L = 2.0 * math.pi / 0.1, 0.05, 64
    got = ff.farfield_3d(u, L, -90.0, 90.0, k, step, step)
    A = ff.fftshift(np.fft.fft(ay, L))
    B = np.fft.fft(bx, L)
    Bm = ff.fftshift(B[(-np.arange(L)) % L])                # conj rows: spectrum at -k
    want = np.outer(np.abs(A) ** 2, np.abs(Bm) ** 2) / L
    assert got.shape == (L, L)
    assert np.allclose(got, want, rtol=1e-10, atol=1e-12 * want.max())


def test_3d_constant_padding_and_reference():
    rng = np.random.default_rng(8)
    n, L = 16, 64
    u = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    ref = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    k, step = 2.0 * math.pi / 0.1, 0.05
    a = ff.farfield_3d(u, L, -90.0, 90.0, k, step, step, reference=ref)
    b = ff.farfield_3d(u - ref, L, -90.0, 90.0, k, step, step)
    assert np.array_equal(a, b)
    c = ff.farfield_3d(u, L, -90.0, 90.0, k, step, step, padding=ff.PAD_CONSTANT)
    # constant padding of a column: entries n.. copy entry 0 -- check one column
    col = np.concatenate([u[:, 3], np.full(L - n, u[0, 3])])
    assert np.allclose(ff.fftshift(np.fft.fft(col)), ff.fftshift(
        np.fft.fft(ff._pad_line(u[:, 3], L, ff.PAD_CONSTANT, n))))
    assert not np.allclose(c, ff.farfield_3d(u, L, -90.0, 90.0, k, step, step))


def test_resize_matrix_blocks():
    m = np.arange(30.0).reshape(5, 6)                     # rows 5, cols 6
    r = ff.resize_matrix(m, 2, 2)                         # dY = 5/3, dX = 2
    # block (0,0): rows 0..1, cols 0..2 ; (1,1): rows 1..3, cols 2..4
    assert r[0, 0] == pytest.approx(m[0:2, 0:3].mean())
    assert r[1, 1] == pytest.approx(m[1:4, 2:5].mean())
    assert r[1, 0] == pytest.approx(m[1:4, 0:3].mean())
    assert ff.resize_matrix(m, 5, 2) is m                 # not smaller in both: unchanged


def test_sources_match_the_oracle_beam():
    """paxpro_b200.sources.GaussianBeam against the oracle's restatement of
    GaussianBeam::get (no GPU needed)."""
    from oracle import pyoracle as po
    from paxpro_b200.sources import GaussianBeam
    from paxpro_b200 import workloads as wl
    n = 64
    dx = wl.step_for_nodes(-500.0, 500.0, n)
    g = po.grid(-500.0, 500.0, dx, -300.0, 300.0, 100.0, 2 * math.pi / 0.1569)
    gb = GaussianBeam(300.0)
    gb.set_wavelength(0.1569)
    x = -500.0 + dx * np.arange(n)
    got = gb.field_3d(x, x)
    want = po.gaussian_beam_3d(g, 0.1569, 300.0)
    assert np.max(np.abs(got - want)) <= 1e-14 * np.max(np.abs(want))
