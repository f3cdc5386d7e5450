"""Regular pose grid: cell-center fractional grid and Fibonacci-sphere directors.

Mirrors the reference ``regular_pose_grid`` (src/string_vext/orientation.py:7-16).
The arithmetic is kept operation-for-operation identical (numpy, float64) so
that centers and directors -- and therefore the field's index layout -- are
bit-identical to the reference's: centers are ((i+.5)/S, (j+.5)/S, (k+.5)/S)
in ``meshgrid(indexing='ij')`` order (i slowest), directors are
z = 1 - 2(k+.5)/n, phi = k*pi*(3 - sqrt(5)).
"""
from __future__ import annotations

import numpy as np


def regular_pose_grid(size: int, orientations: int):
    if size < 2 or orientations < 4:
        raise ValueError("at least two grid cells and four orientations required")
    axis = (np.arange(size, dtype=float) + .5) / size
    centers = np.stack(np.meshgrid(axis, axis, axis, indexing="ij"), axis=-1).reshape(-1, 3)
    z = 1 - 2 * (np.arange(orientations) + .5) / orientations
    phi = np.arange(orientations) * np.pi * (3 - np.sqrt(5))
    directions = np.stack([np.sqrt(1 - z*z) * np.cos(phi),
                           np.sqrt(1 - z*z) * np.sin(phi), z], axis=1)
    return centers, directions


def normalized_directors(axes) -> np.ndarray:
    """Unit directors exactly as the reference native driver forms them
    (src/string_vext/native.py:33-35): ``axes / norm(axes, axis=1)``."""
    axes = np.asarray(axes, dtype=float)
    if (axes.ndim != 2 or axes.shape[1] != 3 or not np.isfinite(axes).all()
            or (np.linalg.norm(axes, axis=1) <= 0).any()):
        raise ValueError("finite nonzero directors required")
    return np.ascontiguousarray(axes / np.linalg.norm(axes, axis=1, keepdims=True))
