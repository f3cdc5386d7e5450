"""GPU String path update and the reference's path-file format.

``run_string`` drives ``vext_string_run`` (csrc/string.cu): the reference
String iteration (native/string/source_code/RC_main.cu:1914-2420) with the
finite-difference forces replaced by the analytic adjoint.  Paths are
(n, 6) arrays of fractional a, b, c and Euler alpha, beta, gamma (radians,
R = Rz(gamma) Ry(beta) Rx(alpha)).

Files keep the reference's formats: output lines are seven ``%.17g`` fields
``a b c alpha beta gamma energy`` (RC_main.cu:2581); an initial path is n
lines of six whitespace-separated numbers (RC_main.cu:1035-1090).
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import _lib


def string_params(**overrides) -> _lib.StringParams:
    p = _lib.StringParams()
    _lib.load().vext_string_default_params(ctypes.byref(p))
    for key, value in overrides.items():
        setattr(p, key, value)
    return p


def run_string(system, path, mode: int = _lib.VEXT_MODE_MIXED, **params):
    """Optimise ``path`` (n, 6) on ``system``; returns (path, energy, result)."""
    path = np.ascontiguousarray(path, dtype=np.float64).copy()
    if path.ndim != 2 or path.shape[1] != 6:
        raise ValueError("path must be (n, 6): a b c alpha beta gamma")
    energy = np.empty(len(path))
    result = _lib.StringResult()
    p = string_params(**params)
    opt = _lib.options(mode)
    _lib.check(_lib.load().vext_string_run(system.handle, len(path), _lib.ptr(path),
                                           _lib.ptr(energy), ctypes.byref(p), ctypes.byref(opt),
                                           ctypes.byref(result)))
    return path, energy, result.as_dict()


def path_selection(case, initial, initial_energy, final, final_energy, direction: int,
                   temperature: float | None = None, mass_g_mol: float | None = None) -> dict:
    """The reference's end-of-run summary (RC_main.cu:2485-2552): hopping
    diffusivity of the final path, log-domain scores of the initial and final
    paths and the chosen one (the initial path when its score is valid and
    higher).  Temperature and guest mass default to the case's."""
    from .tst import choose_initial, diffusivity, hop_length, log_score
    T = float(case["temperature"] if temperature is None else temperature)
    mass = float(case["total_mass"] if mass_g_mol is None else mass_g_mol)
    hop = hop_length(case, direction)
    s_init = log_score(initial, initial_energy, case["cell"], T, mass, hop)
    s_final = log_score(final, final_energy, case["cell"], T, mass, hop)
    use_initial = choose_initial(s_init, s_final)
    return {"diffusivity_final_m2_s": diffusivity(final, final_energy, case["cell"], hop, T, mass),
            "log_d_initial": s_init[1] if s_init[0] else None,
            "log_d_final": s_final[1] if s_final[0] else None,
            "chosen": "initial" if use_initial else "final",
            "peak_initial_K": float(np.max(initial_energy)),
            "peak_final_K": float(np.max(final_energy))}


def write_path(path_file, path, energy) -> None:
    """Seven ``%.17g`` columns per image, as the reference solver writes."""
    lines = [" ".join(f"{v:.17g}" for v in (*row, e)) for row, e in zip(path, energy)]
    Path(path_file).write_text("\n".join(lines) + "\n")


def read_initial(path_file, n_images: int) -> np.ndarray:
    """An initial path: exactly n_images lines, first six numbers of each."""
    lines = [ln for ln in Path(path_file).read_text().splitlines()]
    if len(lines) != n_images:
        raise ValueError(f"initial path has {len(lines)} lines, {n_images} expected")
    return np.array([[float(v) for v in ln.split()[:6]] for ln in lines])


def quaternions_from_euler(euler) -> np.ndarray:
    """Unit quaternions (w, x, y, z) of R = Rz(gamma) Ry(beta) Rx(alpha)."""
    a, b, g = (np.asarray(euler, dtype=float)[:, k] / 2 for k in range(3))
    ca, sa, cb, sb, cg, sg = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(g), np.sin(g)
    return np.stack([cg * cb * ca + sg * sb * sa, cg * cb * sa - sg * sb * ca,
                     cg * sb * ca + sg * cb * sa, sg * cb * ca - cg * sb * sa], 1)


def euler_from_quaternions(q) -> np.ndarray:
    """(alpha, beta, gamma) with R(q) = Rz(gamma) Ry(beta) Rx(alpha), beta in [-pi/2, pi/2]."""
    q = np.asarray(q, dtype=float)
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    r20 = 2 * (x * z - w * y)
    r21 = 2 * (y * z + w * x)
    r22 = 1 - 2 * (x * x + y * y)
    r10 = 2 * (x * y + w * z)
    r00 = 1 - 2 * (y * y + z * z)
    beta = -np.arcsin(np.clip(r20, -1, 1))
    alpha = np.arctan2(r21, r22)
    gamma = np.arctan2(r10, r00)
    return np.stack([alpha, beta, gamma], 1)
