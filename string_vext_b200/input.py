"""Native String ``input.dat`` reader for neutral two-site guests.

Mirrors the reference ``parse_string_input`` (src/string_vext/input.py:11-57):
the same section headers are located, the same validity rules apply (two
neutral sites, neutral numbered framework atoms, positive LJ parameters,
site masses summing to the declared total) and the same case dictionary is
returned, so a case parsed here can be handed to either implementation.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .cell import cell_matrix


def _row_after(lines, prefix):
    for number, line in enumerate(lines):
        if line.startswith(prefix):
            return number + 1
    raise ValueError(f"input section {prefix!r} missing")


def parse_string_input(path) -> dict:
    lines = [line.strip() for line in Path(path).read_text().splitlines()]
    lengths = [float(v) for v in lines[_row_after(lines, "La Lb Lc")].split()[:3]]
    angles = [float(v) for v in lines[_row_after(lines, "Alpha Beta Gamma")].split()[:3]]
    cell = cell_matrix(lengths, angles)
    conditions = [float(v) for v in lines[_row_after(lines, "cutoff(A)")].split()]
    g0 = _row_after(lines, "Number of sites")
    n_guest = int(lines[g0])
    guest = np.array([[float(v) for v in row.split()[:7]]
                      for row in lines[g0 + 2:g0 + 2 + n_guest]])
    f0 = _row_after(lines, "Number of atoms")
    n_frame = int(lines[f0])
    frame = np.array([[float(v) for v in row.split()[:8]]
                      for row in lines[f0 + 2:f0 + 2 + n_frame]])
    if (guest.shape != (2, 7) or frame.shape != (n_frame, 8)
            or len(conditions) < 4 or not np.isfinite(guest).all()
            or not np.isfinite(frame).all() or not np.isfinite(conditions).all()
            or not np.array_equal(frame[:, 0], np.arange(1, n_frame + 1))
            or (guest[:, 5] != 0).any() or (frame[:, 3] != 0).any()
            or (guest[:, 3:5] <= 0).any() or (guest[:, 6] <= 0).any()
            or (frame[:, 1:3] <= 0).any() or conditions[0] <= 0
            or conditions[3] <= 0):
        raise ValueError("invalid or charged two-site String input")
    mass = guest[:, 6]
    total = conditions[2]
    if not np.isclose(mass.sum(), total, rtol=1e-7):
        raise ValueError("guest site masses differ from declared total mass")
    body = guest[:, :3]
    separation = body[1] - body[0]
    bond = np.linalg.norm(separation)
    if bond <= 0:
        raise ValueError("two distinct guest sites required")
    director = separation / bond
    com = (body * mass[:, None]).sum(0) / total
    canonical = np.zeros((2, 3))
    canonical[:, 0] = (body - com) @ director
    return {"cell": cell, "frame_frac": np.mod(frame[:, 5:8], 1),
            "frame_sigma": frame[:, 1], "frame_epsilon": frame[:, 2],
            "guest_xyz": canonical, "guest_sigma": guest[:, 4],
            "guest_epsilon": guest[:, 3], "guest_mass": mass,
            "total_mass": float(total), "temperature": float(conditions[3]),
            "cutoff": float(conditions[0]), "cell_lengths": lengths,
            "cell_angles_deg": angles, "bond_length": float(bond)}


def write_string_input(case: dict, path, n_points: int = 401, delta_frac: float = 1e-4,
                       delta_angle_deg: float = 1.0, direction: int = 1,
                       running_steps: int = 10000) -> None:
    """Write a case in the native ``input.dat`` layout (the inverse of
    ``parse_string_input``), e.g. for handing a synthetic framework to the
    reference CLI or to the String driver."""
    lengths = case["cell_lengths"]
    angles = case["cell_angles_deg"]
    frac = np.asarray(case["frame_frac"], dtype=float)
    lines = ["Nmaxa Nmaxb Nmaxc:", "20 20 20", "La Lb Lc dL",
             f"{lengths[0]:.17g} {lengths[1]:.17g} {lengths[2]:.17g} 0.5",
             "Alpha Beta Gamma",
             f"{angles[0]:.17g} {angles[1]:.17g} {angles[2]:.17g}",
             "cutoff(A) FH_signal Mass(g/mol) Tempearture(K) Running_steps",
             f"{case['cutoff']:.17g} 1 {case['total_mass']:.17g} "
             f"{case['temperature']:.17g} {running_steps}",
             "---------String Calculation Settings---------", "Direction",
             str(direction), "#_of_points delta_frac delta_angle_degree",
             f"{n_points} {delta_frac:.17g} {delta_angle_deg:.17g}",
             "convergence_setting", "default",
             "------------------Adsorbate------------------", "Number of sites", "2",
             "x y z Epsilon Sigma Charge Mass"]
    for site in range(2):
        x = case["guest_xyz"][site]
        lines.append(f"{x[0]:.17g} {x[1]:.17g} {x[2]:.17g} {case['guest_epsilon'][site]:.17g} "
                     f"{case['guest_sigma'][site]:.17g} 0 {case['guest_mass'][site]:.17g}")
    lines += ["------------------Adsorbent-----------------", "Number of atoms",
              str(len(frac)),
              "ID diameter Epsilon Charge mass frac_x frac_y frac_z atom_name"]
    for n, (f, s, e) in enumerate(zip(frac, case["frame_sigma"], case["frame_epsilon"]), 1):
        lines.append(f"{n} {s:.17g} {e:.17g} 0 12.0 {f[0]:.17g} {f[1]:.17g} {f[2]:.17g} X")
    Path(path).write_text("\n".join(lines) + "\n")
