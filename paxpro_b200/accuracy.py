"""Accuracy of a served (FP32) field against its FP64 counterpart.

Two figures per field, the ones the served mode reports beside its speed:

  * relative L2 error of the intensity: ||I - I_ref|| / ||I_ref|| with
    I = |u|^2;
  * intensity-weighted RMS phase error in radians:
    sqrt(sum I_ref * dphi^2 / sum I_ref), dphi = arg(u * conj(u_ref)) in
    (-pi, pi], the phase difference taken point by point, so no 2 pi jumps
    of either field's own phase enter it; dark points, where the phase is
    not defined, weigh nothing.

Only numpy; no device code.
"""
from __future__ import annotations

import numpy as np


def intensity_error(u: np.ndarray, ref: np.ndarray) -> float:
    i = np.abs(np.asarray(u, dtype=np.complex128)) ** 2
    i_ref = np.abs(np.asarray(ref, dtype=np.complex128)) ** 2
    return float(np.linalg.norm(i - i_ref) / np.linalg.norm(i_ref))


def phase_error(u: np.ndarray, ref: np.ndarray) -> float:
    u = np.asarray(u, dtype=np.complex128)
    ref = np.asarray(ref, dtype=np.complex128)
    w = np.abs(ref) ** 2
    dphi = np.angle(u * np.conj(ref))
    return float(np.sqrt(np.sum(w * dphi * dphi) / np.sum(w)))


def field_errors(u: np.ndarray, ref: np.ndarray) -> dict:
    """{"intensity_rel_l2": ..., "phase_rms_rad": ...} of u against ref."""
    return {"intensity_rel_l2": intensity_error(u, ref), "phase_rms_rad": phase_error(u, ref)}
