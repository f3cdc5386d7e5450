"""Transition-state-theory post-processing of a String path: the hopping
diffusivity the reference String program prints and the log-domain score it
uses to choose between the initial and the final path
(native/string/source_code/RC_main.cu:2485-2542, legacy_policy.h:21-53).
The arithmetic runs in the library (vext_tst_*, host code)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _path_arrays(path, energy, cell):
    path = np.asarray(path, dtype=float)
    frac = np.ascontiguousarray(path[:, :3])
    energy = np.ascontiguousarray(energy, dtype=float)
    cell = np.ascontiguousarray(cell, dtype=float)
    if frac.ndim != 2 or len(frac) != len(energy) or cell.shape != (3, 3):
        raise ValueError("path (n, >=3), energy (n,) and a 3x3 cell required")
    return frac, energy, cell


def hop_length(case, direction: int) -> float:
    """The cell length along the transport axis (1 = a, 2 = b, 3 = c), in A."""
    if direction not in (1, 2, 3):
        raise ValueError("direction must be 1, 2 or 3")
    return float(case["cell_lengths"][direction - 1])


def diffusivity(path, energy, cell, hop_A: float, temperature: float,
                mass_g_mol: float) -> float:
    """D0 in m^2/s of a path (rows: fractional a, b, c, ...) with energies in K."""
    frac, energy, cell = _path_arrays(path, energy, cell)
    d0 = ctypes.c_double()
    _lib.check(_lib.load().vext_tst_diffusivity(len(frac), _lib.ptr(frac), _lib.ptr(energy),
                                                _lib.ptr(cell), float(hop_A),
                                                float(temperature), float(mass_g_mol),
                                                ctypes.byref(d0)))
    return d0.value


def log_score(path, energy, cell, temperature: float, mass_g_mol: float,
              hop_A: float) -> tuple[bool, float]:
    """(valid, log D) with the shifted-energy trapezoid in log space."""
    frac, energy, cell = _path_arrays(path, energy, cell)
    valid, logd = ctypes.c_int(), ctypes.c_double()
    _lib.check(_lib.load().vext_tst_log_score(len(frac), _lib.ptr(frac), _lib.ptr(energy),
                                              _lib.ptr(cell), float(temperature),
                                              float(mass_g_mol), float(hop_A),
                                              ctypes.byref(valid), ctypes.byref(logd)))
    return bool(valid.value), logd.value


def choose_initial(initial: tuple[bool, float], final: tuple[bool, float]) -> bool:
    """The reference keeps the initial path when its score is valid and higher
    than the final path's (or the final score is invalid)."""
    return initial[0] and (not final[0] or initial[1] > final[1])
