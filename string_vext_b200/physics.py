"""Case validation and small host-side physics helpers.

Mirrors the reference's ``validate_case``, ``body_offsets`` and
``marginal_energy`` (src/string_vext/physics.py:16-40, 88-90, 126-130):
same rules, same error messages, same formulas.  Everything heavy runs in
the CUDA library; these helpers only prepare inputs and check outputs.
"""
from __future__ import annotations

import numpy as np


def validate_case(case) -> None:
    cell = np.asarray(case["cell"], dtype=float)
    frame = np.asarray(case["frame_frac"], dtype=float)
    if (cell.shape != (3, 3) or not np.isfinite(cell).all() or np.linalg.det(cell) <= 0
            or frame.ndim != 2 or frame.shape[1] != 3 or not len(frame)
            or not np.isfinite(frame).all()):
        raise ValueError("invalid triclinic framework")
    for key in ("frame_sigma", "frame_epsilon"):
        values = np.asarray(case[key], dtype=float)
        if values.shape != (len(frame),) or not np.isfinite(values).all() or (values <= 0).any():
            raise ValueError("invalid framework LJ parameters")
    for key in ("guest_sigma", "guest_epsilon", "guest_mass"):
        values = np.asarray(case[key], dtype=float)
        if values.shape != (2,) or not np.isfinite(values).all() or (values <= 0).any():
            raise ValueError("invalid two-site guest")
    body = np.asarray(case["guest_xyz"], dtype=float)
    if body.shape != (2, 3) or not np.isfinite(body).all() or not np.allclose(body[:, 1:], 0):
        raise ValueError("guest must have a two-site body x-axis")
    if not np.isclose(sum(case["guest_mass"]), case["total_mass"], rtol=1e-6):
        raise ValueError("guest mass mismatch")
    if (not np.isfinite([case["cutoff"], case["temperature"]]).all()
            or min(case["cutoff"], case["temperature"]) <= 0):
        raise ValueError("invalid cutoff/temperature")


def require_identical_sites(case) -> None:
    """Neighbour reuse needs two identical sites (src/string_vext/neighbor.py:12-16)."""
    sigma = np.asarray(case["guest_sigma"], dtype=float)
    epsilon = np.asarray(case["guest_epsilon"], dtype=float)
    if (sigma.shape != (2,) or epsilon.shape != (2,)
            or sigma[0] != sigma[1] or epsilon[0] != epsilon[1]):
        raise ValueError("exact neighbor reuse requires identical two-site LJ parameters")


def body_offsets(case) -> np.ndarray:
    """Signed COM-relative offsets of the two sites along the body x axis."""
    xyz = np.asarray(case["guest_xyz"], dtype=float)
    mass = np.asarray(case["guest_mass"], dtype=float)
    com = (xyz * mass[:, None]).sum(0) / case["total_mass"]
    return xyz[:, 0] - com[0]


def marginal_energy(energies, temperature) -> np.ndarray:
    """-T (logsumexp(-E/T) - log n) over the last axis (host reference of the
    quantity the field epilogue computes on the device)."""
    from scipy.special import logsumexp
    energy = np.asarray(energies, dtype=float)
    if not np.isfinite(energy).all() or not np.isfinite(temperature) or temperature <= 0:
        raise ValueError("finite angular energies and positive temperature required")
    return -temperature * (logsumexp(-energy / temperature, axis=-1) - np.log(energy.shape[-1]))
