"""Exact triclinic Vext fields on the GPU: ``calculate_vext`` and the CLI.

``calculate_vext(case, size, orientations)`` returns the reference's output
dictionary (src/string_vext/vext.py:21-43): ``orientation_K``,
``marginal_K``, ``site_K``, ``axes``, ``cell_matrix``, ``atom_fractional``,
``framework_sigma_A``, ``framework_epsilon_K``, ``grid``.  Centers and
directors come from ``regular_pose_grid`` with the reference's arithmetic,
so the index layout is bit-identical; energies, marginal, site field and
grid come from one call of the CUDA library (``vext_field``): region lists
built on the GPU, no host kd-tree and no CSR.

The CLI keeps the reference's command contract (src/string_vext/vext.py:
46-84): ``--input --output --size --orientations --kernel``; it never
overwrites -- an existing NPZ or provenance record is a ``FileExistsError``
and both files are created exclusively; the provenance record carries the
SHA-256 of input, output and library.  ``--kernel`` names the build of this
library to load (default: the in-tree one).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import tempfile
from pathlib import Path

import numpy as np

from . import _lib
from .input import parse_string_input
from .orientation import normalized_directors, regular_pose_grid


def calculate_vext(case: dict, size: int = 60, orientations: int = 64,
                   mode: int = _lib.VEXT_MODE_MIXED, return_stats: bool = False):
    """The Vext field of ``case`` on a ``size``^3 grid x ``orientations``
    Fibonacci directors, in the reference's output layout."""
    from .system import VextSystem
    _, axes = regular_pose_grid(size, orientations)
    with VextSystem(case) as system:
        out = system.field(size, normalized_directors(axes), mode=mode, orientation=True,
                           marginal=True, site=True, grid=True)
        stats = system.last_stats
    result = {"orientation_K": out["orientation_K"], "marginal_K": out["marginal_K"],
              "site_K": out["site_K"], "axes": axes.astype(np.float32),
              "cell_matrix": np.asarray(case["cell"], dtype=np.float64),
              "atom_fractional": np.asarray(case["frame_frac"], dtype=np.float64),
              "framework_sigma_A": np.asarray(case["frame_sigma"], dtype=np.float64),
              "framework_epsilon_K": np.asarray(case["frame_epsilon"], dtype=np.float64),
              "grid": out["grid"]}
    for name, value in result.items():
        if not np.isfinite(value).all():
            raise ValueError(f"nonfinite Vext output ({name})")
    return (result, stats) if return_stats else result


def _sha256(path: Path) -> str:
    digest = hashlib.sha256()
    with open(path, "rb") as handle:
        for block in iter(lambda: handle.read(1 << 20), b""):
            digest.update(block)
    return digest.hexdigest()


def _publish_npz(destination: Path, arrays: dict) -> None:
    """Write an NPZ next to ``destination`` under a fresh private name, then
    hard-link it into place: the link fails if ``destination`` appeared in
    the meantime, so an existing file is never replaced and a reader never
    sees a partial archive."""
    destination.parent.mkdir(parents=True, exist_ok=True)
    handle, scratch = tempfile.mkstemp(prefix=destination.name + ".", suffix=".part",
                                       dir=destination.parent)
    try:
        with os.fdopen(handle, "wb") as stream:
            np.savez_compressed(stream, **arrays)
            stream.flush()
            os.fsync(stream.fileno())
        os.link(scratch, destination)
    finally:
        os.unlink(scratch)


def provenance(input_path: Path, output_path: Path, library: Path, size: int,
               orientations: int, case: dict, fp64: bool) -> dict:
    return {"input": str(input_path.resolve()), "input_sha256": _sha256(input_path),
            "output_sha256": _sha256(output_path), "kernel_sha256": _sha256(library),
            "size": size, "orientations": orientations,
            "energy_mode": "exact_triclinic_LJ_b200_" + ("fp64" if fp64 else "mixed"),
            "cell_lengths_A": case["cell_lengths"], "cell_angles_deg": case["cell_angles_deg"],
            "guest_sigma_A": case["guest_sigma"].tolist(),
            "guest_epsilon_K": case["guest_epsilon"].tolist()}


def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__,
                                     formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("--input", type=Path, required=True, help="native String input.dat")
    parser.add_argument("--output", type=Path, required=True, help="new NPZ destination")
    parser.add_argument("--size", type=int, default=60, help="grid points per axis")
    parser.add_argument("--orientations", type=int, default=64)
    parser.add_argument("--kernel", type=Path, default=None,
                        help="build of libvext_b200.so to load (default: the in-tree one)")
    parser.add_argument("--fp64", action="store_true", help="all pairs in FP64")
    args = parser.parse_args(argv)
    record_path = args.output.with_suffix(".json")
    if args.output.exists() or record_path.exists():
        raise FileExistsError("Vext output or provenance record already exists")
    library = Path(args.kernel) if args.kernel else _lib.LIB_PATH
    _lib.load(library)
    case = parse_string_input(args.input)
    mode = _lib.VEXT_MODE_FP64 if args.fp64 else _lib.VEXT_MODE_MIXED
    _publish_npz(args.output, calculate_vext(case, args.size, args.orientations, mode=mode))
    record = provenance(args.input, args.output, library, args.size, args.orientations, case,
                        args.fp64)
    with record_path.open("x") as handle:
        handle.write(json.dumps(record, indent=2) + "\n")
    print(json.dumps(record, sort_keys=True))


if __name__ == "__main__":
    main()
