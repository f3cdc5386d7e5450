"""Exact triclinic Vext fields on the GPU: ``calculate_vext`` and the CLI.

Mirrors the reference's ``calculate_vext`` / ``main`` (src/string_vext/vext.py:
21-84): same arguments, same output dictionary (``orientation_K``,
``marginal_K``, ``site_K``, ``axes``, ``cell_matrix``, ``atom_fractional``,
``framework_sigma_A``, ``framework_epsilon_K``, ``grid``), same NPZ +
provenance-JSON writer with exclusive creation.  The pose grid and directors
come from ``regular_pose_grid`` with the reference's own arithmetic, so the
index layout is bit-identical; the energies, marginal, site field and grid
are computed by the CUDA library in one call (no kd-tree, no CSR).

With ``kernel=`` a path to an ``evaluate_reused_neighbors`` library, the
reference's CSR route (``NativeReusePotential``) is taken instead, so any
build of the reference kernel -- or this project's drop-in -- can be used.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
from pathlib import Path

import numpy as np

from . import _lib
from .input import parse_string_input
from .orientation import normalized_directors, regular_pose_grid
from .physics import marginal_energy


def calculate_vext(case: dict, size: int = 60, orientations: int = 64, kernel=None,
                   mode: int = _lib.VEXT_MODE_MIXED, return_stats: bool = False):
    centers, axes = regular_pose_grid(size, orientations)
    if kernel is not None:
        from .native import NativeReusePotential
        from .system import VextSystem
        energy = NativeReusePotential(case, kernel).evaluate(centers, axes)
        marginal = marginal_energy(energy, case["temperature"])
        with VextSystem(case) as system:
            site = system.field(size, normalized_directors(axes), orientation=False,
                                site=True, mode=_lib.VEXT_MODE_FP64)["site_K"]
        orientation_K = energy.T.reshape(orientations, size, size, size).astype(np.float32)
        marginal_K = marginal.reshape(size, size, size).astype(np.float32)
        stats = None
    else:
        from .system import VextSystem
        with VextSystem(case) as system:
            out = system.field(size, normalized_directors(axes), mode=mode, orientation=True,
                               marginal=True, site=True, grid=True)
            stats = system.last_stats
        orientation_K, marginal_K, site = out["orientation_K"], out["marginal_K"], out["site_K"]
    result = {
        "orientation_K": orientation_K,
        "marginal_K": marginal_K,
        "site_K": site,
        "axes": axes.astype(np.float32),
        "cell_matrix": np.asarray(case["cell"], dtype=np.float64),
        "atom_fractional": np.asarray(case["frame_frac"], dtype=np.float64),
        "framework_sigma_A": np.asarray(case["frame_sigma"], dtype=np.float64),
        "framework_epsilon_K": np.asarray(case["frame_epsilon"], dtype=np.float64),
    }
    result["grid"] = np.arcsinh(result["marginal_K"] / 1000).astype(np.float32)
    if any(not np.isfinite(value).all() for value in result.values()):
        raise ValueError("nonfinite Vext output")
    return (result, stats) if return_stats else result


def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--input", type=Path, required=True, help="native String input.dat")
    parser.add_argument("--output", type=Path, required=True, help="new NPZ destination")
    parser.add_argument("--size", type=int, default=60, help="grid points per axis")
    parser.add_argument("--orientations", type=int, default=64)
    parser.add_argument("--kernel", type=Path, default=None,
                        help="optional evaluate_reused_neighbors library (CSR route)")
    parser.add_argument("--fp64", action="store_true", help="all pairs in FP64")
    args = parser.parse_args(argv)
    record_path = args.output.with_suffix(".json")
    if args.output.exists() or record_path.exists():
        raise FileExistsError("Vext output or provenance record already exists")
    case = parse_string_input(args.input)
    mode = _lib.VEXT_MODE_FP64 if args.fp64 else _lib.VEXT_MODE_MIXED
    fields = calculate_vext(case, args.size, args.orientations, args.kernel, mode=mode)
    args.output.parent.mkdir(parents=True, exist_ok=True)
    temporary = args.output.with_suffix(".npz.tmp")
    try:
        with temporary.open("xb") as handle:
            np.savez_compressed(handle, **fields)
        os.link(temporary, args.output)
    finally:
        temporary.unlink(missing_ok=True)
    library = Path(args.kernel) if args.kernel else _lib.LIB_PATH
    record = {"input": str(args.input.resolve()),
              "input_sha256": hashlib.sha256(args.input.read_bytes()).hexdigest(),
              "output_sha256": hashlib.sha256(args.output.read_bytes()).hexdigest(),
              "kernel_sha256": hashlib.sha256(library.read_bytes()).hexdigest(),
              "size": args.size, "orientations": args.orientations,
              "energy_mode": "exact_triclinic_LJ_b200_" + ("fp64" if args.fp64 else "mixed"),
              "cell_lengths_A": case["cell_lengths"],
              "cell_angles_deg": case["cell_angles_deg"],
              "guest_sigma_A": case["guest_sigma"].tolist(),
              "guest_epsilon_K": case["guest_epsilon"].tolist()}
    with record_path.open("x") as handle:
        json.dump(record, handle, indent=2)
        handle.write("\n")
    print(json.dumps(record, sort_keys=True))


if __name__ == "__main__":
    main()
