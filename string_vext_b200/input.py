"""The native String ``input.dat`` layout, for neutral two-site guests.

The file is a sequence of labelled blocks: a label line (``La Lb Lc dL``,
``Alpha Beta Gamma``, ``cutoff(A) ...``, ``Number of sites``, ``Number of
atoms`` ...) followed by its value lines.  A site block is a count line, a
column header, then one ``x y z epsilon sigma charge mass`` row per site; a
framework block is a count line, a column header, then one ``id sigma
epsilon charge mass frac_a frac_b frac_c [name]`` row per atom (the layout the
reference String program reads, native/string/source_code/RC_main.cu:282-390).

``parse_string_input`` returns the reference's case dictionary and enforces
its acceptance rules with its messages (src/string_vext/input.py:11-57): two
neutral sites with positive LJ parameters and masses summing to the declared
total, neutral framework atoms numbered 1..N with positive sigma and
epsilon, a positive cutoff and temperature.  The guest is stored canonically:
both sites on the body x axis at their signed distance from the centre of
mass, which fixes the site offsets the energy kernels use.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .cell import cell_matrix

#: Label prefixes of the blocks the parser reads.
LENGTHS, ANGLES, CONDITIONS = "La Lb Lc", "Alpha Beta Gamma", "cutoff(A)"
SITES, ATOMS = "Number of sites", "Number of atoms"

_REJECT = "invalid or charged two-site String input"


class _Blocks:
    """Value lines of an input file addressed by the label that precedes them."""

    def __init__(self, text: str):
        self.lines = [line.strip() for line in text.splitlines()]
        self.start = {}
        for number, line in enumerate(self.lines):
            for label in (LENGTHS, ANGLES, CONDITIONS, SITES, ATOMS):
                if line.startswith(label) and label not in self.start:
                    self.start[label] = number + 1

    def first(self, label: str) -> int:
        if label not in self.start:
            raise ValueError(f"input section {label!r} missing")
        return self.start[label]

    def numbers(self, row: int, width: int | None = None) -> list[float]:
        fields = self.lines[row].split() if row < len(self.lines) else []
        return [float(v) for v in (fields if width is None else fields[:width])]

    def table(self, label: str, width: int) -> np.ndarray:
        """The counted table of a block: count line, header line, rows."""
        at = self.first(label)
        count = int(self.lines[at])
        if count < 0:
            raise ValueError(_REJECT)
        rows = [self.numbers(at + 2 + k, width) for k in range(count)]
        if any(len(r) != width for r in rows):
            raise ValueError(_REJECT)
        return np.array(rows, dtype=float).reshape(count, width)


def _accept(guest: np.ndarray, frame: np.ndarray, conditions: list[float]) -> bool:
    numbered = np.array_equal(frame[:, 0], np.arange(1, len(frame) + 1))
    return (guest.shape == (2, 7) and len(frame) >= 1 and len(conditions) >= 4 and numbered
            and all(np.isfinite(a).all() for a in (guest, frame, np.array(conditions)))
            and not guest[:, 5].any() and not frame[:, 3].any()
            and (guest[:, 3:5] > 0).all() and (guest[:, 6] > 0).all()
            and (frame[:, 1:3] > 0).all() and conditions[0] > 0 and conditions[3] > 0)


def parse_string_input(path) -> dict:
    blocks = _Blocks(Path(path).read_text())
    lengths = blocks.numbers(blocks.first(LENGTHS), 3)
    angles = blocks.numbers(blocks.first(ANGLES), 3)
    cell = cell_matrix(lengths, angles)
    conditions = blocks.numbers(blocks.first(CONDITIONS))   # rc, FH flag, mass, T, steps
    guest = blocks.table(SITES, 7)
    frame = blocks.table(ATOMS, 8)
    if not _accept(guest, frame, conditions):
        raise ValueError(_REJECT)
    cutoff, total, temperature = conditions[0], conditions[2], conditions[3]
    mass = guest[:, 6]
    if not np.isclose(mass.sum(), total, rtol=1e-7):
        raise ValueError("guest site masses differ from declared total mass")
    xyz = guest[:, :3]
    axis = xyz[1] - xyz[0]
    bond = np.linalg.norm(axis)
    if bond <= 0:
        raise ValueError("two distinct guest sites required")
    centre = (xyz * mass[:, None]).sum(0) / total
    body = np.zeros((2, 3))
    body[:, 0] = (xyz - centre) @ (axis / bond)
    return {"cell": cell, "frame_frac": np.mod(frame[:, 5:8], 1),
            "frame_sigma": frame[:, 1], "frame_epsilon": frame[:, 2],
            "guest_xyz": body, "guest_sigma": guest[:, 4],
            "guest_epsilon": guest[:, 3], "guest_mass": mass,
            "total_mass": float(total), "temperature": float(temperature),
            "cutoff": float(cutoff), "cell_lengths": lengths,
            "cell_angles_deg": angles, "bond_length": float(bond)}


def write_string_input(case: dict, path, n_points: int = 401, delta_frac: float = 1e-4,
                       delta_angle_deg: float = 1.0, direction: int = 1,
                       running_steps: int = 10000) -> None:
    """Write a case in the native ``input.dat`` layout (the inverse of
    ``parse_string_input``), e.g. for handing a synthetic framework to the
    reference String program or its Python CLI."""
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
