"""Triclinic cell matrix (row vectors; Cartesian = fractional @ cell).

Mirrors the reference ``cell_matrix`` (src/string_vext/cell.py:7-29): the a
vector lies along x, b in the xy plane, c from the three cosines; the same
validity checks raise ``ValueError`` with the same messages.  The formula has
to be identical because the cell defines the image lattice every energy is
summed over.
"""
from __future__ import annotations

import numpy as np


def cell_matrix(lengths, angles_deg) -> np.ndarray:
    lengths = np.asarray(lengths, dtype=float)
    angles = np.asarray(angles_deg, dtype=float)
    if (lengths.shape != (3,) or angles.shape != (3,)
            or not np.isfinite(lengths).all() or not np.isfinite(angles).all()
            or (lengths <= 0).any() or (angles <= 0).any() or (angles >= 180).any()):
        raise ValueError("three positive lengths and three angles in (0, 180) required")
    alpha, beta, gamma = np.deg2rad(angles)
    a, b, c = lengths
    sin_gamma = np.sin(gamma)
    if abs(sin_gamma) < 1e-10:
        raise ValueError("singular triclinic cell")
    cx = c * np.cos(beta)
    cy = c * (np.cos(alpha) - np.cos(beta) * np.cos(gamma)) / sin_gamma
    cz2 = c * c - cx * cx - cy * cy
    if cz2 <= 0:
        raise ValueError("nonphysical triclinic cell")
    matrix = np.array([[a, 0., 0.],
                       [b * np.cos(gamma), b * sin_gamma, 0.],
                       [cx, cy, np.sqrt(cz2)]])
    if not np.isfinite(matrix).all() or np.linalg.det(matrix) <= 0:
        raise ValueError("invalid cell determinant")
    return matrix


def valid_cell(lengths, angles_deg) -> bool:
    """True when ``cell_matrix`` accepts the six parameters."""
    try:
        cell_matrix(lengths, angles_deg)
    except ValueError:
        return False
    return True
