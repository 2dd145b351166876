"""CPU restatement of post::FarField (the far-field post-processing module).

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the product package.

Follows src/farFieldPost.cpp step by step, with numpy's FFT (pocketfft)
standing in for FFTW / arma::fft (unnormalised forward transform,
exp(-2 pi i jk/L)):

  * 2-D (`result(solver, arma::vec&)`, :22-62): the exit field centred in a
    line of `pad_length` entries filled with the pad value
    (ParaxialSimulation::padExitField, include/paraxialSimulation.hpp:174),
    or the bare field when `pad_length` is below its length; |FFT| /
    sqrt(L); fftshift (:64-74, the halves swapped, the middle entry of an odd
    length left in place); the angular crop of reduceArray (:103-111) along x;
  * 3-D (`result(solver, arma::mat&)`, :141-247): L = max(pad_length, rows,
    cols); the field minus the reference (when set); FFT of every column
    zero-padded to L (constant padding: entries from N on copy entry 0,
    :314-321), fftshift, crop along y; then FFT of every row of that, taken
    as Armadillo's `.t()` of a complex row -- the conjugate transpose --
    padded to L the same way, fftshift, crop along x, |.|^2 / L; finally
    PostProcessingModule::resizeMatrix (src/postProcessing.cpp:29-49) when
    export dimensions are set.

The angle-to-index map is farFieldAngleToIndx (:78-101). Linear-fit
padding (:265-312, GSL) is not restated: the reference marks it untested
and the device path does not provide it.

No reference test holds far-field values; the FFT is pocketfft, not FFTW,
so this restatement is "parity unpinned" beyond the FFT's own accuracy.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

PI = math.acos(-1.0)
PAD_ZERO, PAD_LINEAR_FIT, PAD_CONSTANT = 0, 1, 2


def angle_to_index(angle: float, size: int, wavenumber: float, step: float) -> int:
    """farFieldAngleToIndx (src/farFieldPost.cpp:78-101)."""
    angle_rad = angle * PI / 180.0
    n = int(size * wavenumber * step * math.sin(angle_rad) / (2.0 * PI))  # truncation
    if abs(n) >= size // 2:
        return size - 1 if angle > 0.0 else 0
    return n + size // 2


def fftshift(a: np.ndarray) -> np.ndarray:
    """FarField::fftshift (:64-74): swap entry i with i + N/2 for i < N/2."""
    out = a.copy()
    h = a.shape[0] // 2
    out[:h] = a[h:2 * h]
    out[h:2 * h] = a[:h]
    return out


def farfield_2d(u: np.ndarray, pad_length: int, phi_min: float, phi_max: float,
                wavenumber: float, dx: float, pad_value: complex = 0.0) -> np.ndarray:
    """FarField::result for a 2-D solver: the exit field u (length N)."""
    n = u.shape[0]
    if pad_length < n:
        padded = u.astype(np.complex128).copy()
    else:
        padded = np.full(pad_length, complex(pad_value), dtype=np.complex128)
        start = pad_length // 2 - n // 2
        padded[start:start + n] = u
    ft = np.fft.fft(padded)
    res = np.abs(ft) / math.sqrt(ft.shape[0])
    res = fftshift(res)
    lo = angle_to_index(phi_min, res.shape[0], wavenumber, dx)
    hi = angle_to_index(phi_max, res.shape[0], wavenumber, dx)
    return res[lo:hi + 1].copy()


def _pad_line(v: np.ndarray, L: int, padding: int, n_nodes: int) -> np.ndarray:
    pad = np.zeros(L, dtype=np.complex128)
    pad[:v.shape[0]] = v
    if padding == PAD_CONSTANT:
        pad[n_nodes:] = pad[0]
    elif padding != PAD_ZERO:
        raise ValueError("linear-fit padding is not restated")
    return pad


def resize_matrix(orig: np.ndarray, rows: int, cols: int) -> np.ndarray:
    """PostProcessingModule::resizeMatrix (src/postProcessing.cpp:29-49):
    overlapping blocks, inclusive bounds truncated from doubles, the mean of
    the column means."""
    if rows >= orig.shape[0] or cols >= orig.shape[1]:
        return orig
    dX = orig.shape[1] / (cols + 1.0)
    dY = orig.shape[0] / (rows + 1.0)
    out = np.empty((rows, cols))
    for i in range(cols):
        c0, c1 = int(i * dX), int((i + 1) * dX)
        for j in range(rows):
            r0, r1 = int(j * dY), int((j + 1) * dY)
            out[j, i] = orig[r0:r1 + 1, c0:c1 + 1].mean(axis=0).mean()
    return out


def farfield_3d(u: np.ndarray, pad_length: int, phi_min: float, phi_max: float,
                wavenumber: float, dx: float, dy: float,
                reference: Optional[np.ndarray] = None, padding: int = PAD_ZERO,
                export_rows: int = 0, export_cols: int = 0) -> np.ndarray:
    """FarField::result for a 3-D solver: u is the (rows=y, cols=x) exit field."""
    rows, cols = u.shape
    L = max(pad_length, rows, cols)
    sol = u.astype(np.complex128)
    if reference is not None:
        sol = sol - reference
    n_nodes = cols  # nodeNumberTransverse
    lo = angle_to_index(phi_min, L, wavenumber, dy)
    hi = angle_to_index(phi_max, L, wavenumber, dy)
    if hi < lo:
        raise ValueError("empty angular range")
    nrows = hi - lo + 1
    temp = np.zeros((nrows, cols), dtype=np.complex128)
    for c in range(cols):
        ft = fftshift(np.fft.fft(_pad_line(sol[:, c], L, padding, n_nodes)))
        temp[:, c] = ft[lo:hi + 1]
    lo_x = angle_to_index(phi_min, L, wavenumber, dx)
    hi_x = angle_to_index(phi_max, L, wavenumber, dx)
    if hi_x < lo_x:
        raise ValueError("empty angular range")
    res = np.empty((nrows, hi_x - lo_x + 1))
    for r in range(nrows):
        row = np.conj(temp[r, :])  # Armadillo's .t() of a complex row
        ft = fftshift(np.fft.fft(_pad_line(row, L, padding, n_nodes)))
        res[r, :] = np.abs(ft[lo_x:hi_x + 1]) ** 2 / L
    if export_rows and export_cols:
        res = resize_matrix(res, export_rows, export_cols)
    return res
