"""Seeded synthetic frameworks and guests for the five benchmark workloads.

There is no dataset: every framework is drawn from ``numpy.random.default_rng``
with a fixed seed and a fixed draw order, documented per workload below, so
any machine regenerates bit-identical inputs.  The returned dictionaries use
the reference's case layout (src/string_vext/input.py:49-55): ``cell`` (row
vectors), ``frame_frac``, ``frame_sigma``, ``frame_epsilon``, ``guest_xyz``
(two sites on the body x axis, center of mass at the origin),
``guest_sigma``, ``guest_epsilon``, ``guest_mass``, ``total_mass``,
``temperature``, ``cutoff``, ``cell_lengths``, ``cell_angles_deg``,
``bond_length``.

Workloads (sizes per the benchmark definition):

* ``small_field``  -- 15 x 15 x 10 A, gamma 120, 64 atoms (seed 0), per-atom
  eps U(20, 60) K, sigma U(2.5, 3.8) A; guest 98 K / 3.75 A / bond 1.54 A;
  cutoff 12.0 A; 20^3 grid x 64 directors.
* ``full_field``   -- 37 x 37 x 3.6 A, gamma 119.993, 600 atoms (seed 1),
  layered (z near 0 or 0.5), 4-type table; guest 85 K / 3.685 A / 1.33 A;
  cutoff 12.8 A; 60^3 x 64.
* ``skewed_field`` -- 28 x 31 x 24 A, angles 75/85/110, 3000 uniform atoms
  (seed 2), 4-type table; guest 98 K / 3.75 A / 1.54 A; cutoff 12.8 A; 60^3 x 64.
* ``string_path``  -- framework of ``small_field``; a 64-image path along the
  fractional c axis at (0.25, 0.25) with random unit quaternions (seed 3), and
  a 65536-pose random batch.
* ``batch``        -- 50 frameworks (seed 4), two guests each -> 100 fields.
"""
from __future__ import annotations

import numpy as np

from .cell import cell_matrix, valid_cell

#: (epsilon/kB in K, sigma in A) of the four framework atom types.
TYPE_TABLE = np.array([[52.8, 3.43], [34.7, 3.26], [30.2, 3.12], [22.1, 2.57]])

#: (epsilon/kB K, sigma A, bond A) of the two benchmark guests.
GUEST_A = (98.0, 3.75, 1.54)
GUEST_B = (85.0, 3.685, 1.33)

SITE_MASS = 15.0
TEMPERATURE = 298.0


def make_case(lengths, angles, frac, sigma, epsilon, guest, cutoff,
              temperature: float = TEMPERATURE) -> dict:
    """Assemble a case dictionary; ``guest`` = (epsilon K, sigma A, bond A)."""
    eps_g, sig_g, bond = (float(v) for v in guest)
    cell = cell_matrix(lengths, angles)
    body = np.zeros((2, 3))
    body[:, 0] = (-bond / 2, bond / 2)
    return {"cell": cell, "frame_frac": np.mod(np.asarray(frac, dtype=float), 1),
            "frame_sigma": np.asarray(sigma, dtype=float),
            "frame_epsilon": np.asarray(epsilon, dtype=float),
            "guest_xyz": body, "guest_sigma": np.array([sig_g, sig_g]),
            "guest_epsilon": np.array([eps_g, eps_g]),
            "guest_mass": np.array([SITE_MASS, SITE_MASS]),
            "total_mass": 2 * SITE_MASS, "temperature": float(temperature),
            "cutoff": float(cutoff), "cell_lengths": [float(v) for v in lengths],
            "cell_angles_deg": [float(v) for v in angles], "bond_length": bond}


def small_field() -> dict:
    """Draw order (seed 0): frac (64, 3) U[0,1); eps (64,) U(20, 60); sigma (64,) U(2.5, 3.8)."""
    rng = np.random.default_rng(0)
    frac = rng.random((64, 3))
    eps = rng.uniform(20.0, 60.0, 64)
    sig = rng.uniform(2.5, 3.8, 64)
    return make_case([15.0, 15.0, 10.0], [90.0, 90.0, 120.0], frac, sig, eps, GUEST_A, 12.0)


def full_field() -> dict:
    """Draw order (seed 1): xy (600, 2) U[0,1); layer (600,) integers{0,1};
    jitter (600,) N(0, 0.02); type (600,) integers{0..3}.  z = 0.5*layer + jitter."""
    rng = np.random.default_rng(1)
    xy = rng.random((600, 2))
    layer = rng.integers(0, 2, 600)
    jitter = rng.normal(0.0, 0.02, 600)
    kind = rng.integers(0, 4, 600)
    frac = np.column_stack([xy, 0.5 * layer + jitter])
    return make_case([37.0, 37.0, 3.6], [90.0, 90.0, 119.993], frac,
                     TYPE_TABLE[kind, 1], TYPE_TABLE[kind, 0], GUEST_B, 12.8)


def skewed_field() -> dict:
    """Draw order (seed 2): frac (3000, 3) U[0,1); type (3000,) integers{0..3}."""
    rng = np.random.default_rng(2)
    frac = rng.random((3000, 3))
    kind = rng.integers(0, 4, 3000)
    return make_case([28.0, 31.0, 24.0], [75.0, 85.0, 110.0], frac,
                     TYPE_TABLE[kind, 1], TYPE_TABLE[kind, 0], GUEST_A, 12.8)


def random_quaternions(rng, n: int) -> np.ndarray:
    """Uniform unit quaternions (w, x, y, z): normalised 4-D Gaussian draws."""
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def string_path(n_images: int = 64):
    """Draw order (seed 3): path quaternions (n_images, 4) N(0,1) normalised;
    then the random batch: centers (65536, 3) U[0,1) fractional, quaternions
    (65536, 4) N(0,1) normalised.  Returns (case, path_frac, path_quat,
    batch_frac, batch_quat)."""
    case = small_field()
    rng = np.random.default_rng(3)
    t = np.linspace(0.0, 1.0, n_images)
    path_frac = np.column_stack([np.full(n_images, 0.25), np.full(n_images, 0.25), t])
    path_quat = random_quaternions(rng, n_images)
    batch_frac = rng.random((65536, 3))
    batch_quat = random_quaternions(rng, 65536)
    return case, path_frac, path_quat, batch_frac, batch_quat


def batch_frameworks(n_frameworks: int = 50):
    """Draw order (seed 4), per framework in turn: n = round(exp(U(ln 100, ln 4000)));
    lengths (3,) U(10, 45); angles (3,) U(60, 120), angles redrawn until the
    cell is valid; frac (n, 3) U[0,1); type (n,) integers{0..3}.  Each framework
    is paired with both guests (cutoff 12.8 A).  Returns a list of cases
    ordered framework-major, guest A then guest B."""
    rng = np.random.default_rng(4)
    cases = []
    for _ in range(n_frameworks):
        n = int(round(np.exp(rng.uniform(np.log(100.0), np.log(4000.0)))))
        lengths = rng.uniform(10.0, 45.0, 3)
        angles = rng.uniform(60.0, 120.0, 3)
        while not valid_cell(lengths, angles):
            angles = rng.uniform(60.0, 120.0, 3)
        frac = rng.random((n, 3))
        kind = rng.integers(0, 4, n)
        for guest in (GUEST_A, GUEST_B):
            cases.append(make_case(lengths, angles, frac, TYPE_TABLE[kind, 1],
                                   TYPE_TABLE[kind, 0], guest, 12.8))
    return cases


def string_paths_batch(cases, n_paths: int = 100, seed: int = 5):
    """Random String paths for the batched forward+adjoint workload: path p
    uses ``cases[p % len(cases)]``; draw order (seed 5) per path: length
    integers[32, 96]; start and end (2, 3) U[0,1) fractional; quaternions
    (length, 4) N(0,1) normalised.  Returns a list of (case_index, frac, quat)."""
    rng = np.random.default_rng(seed)
    paths = []
    for p in range(n_paths):
        n = int(rng.integers(32, 97))
        ends = rng.random((2, 3))
        t = np.linspace(0.0, 1.0, n)[:, None]
        frac = ends[0] + t * (ends[1] - ends[0])
        quat = random_quaternions(rng, n)
        paths.append((p % len(cases), frac, quat))
    return paths


WORKLOADS = {"small_field": (small_field, 20), "full_field": (full_field, 60),
             "skewed_field": (skewed_field, 60)}
