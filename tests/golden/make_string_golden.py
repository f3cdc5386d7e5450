"""Golden String paths produced by the reference String solver itself.

The reference's String program (native/string/source_code/RC_main.cu with
global.h, unchanged) is built from its sources by

    make -C oracle string REF=<reference checkout>      # -> oracle/_ref/string_triclinic_cuda

and then, on a machine with a CUDA GPU,

    python tests/golden/make_string_golden.py run --out <dir>

writes each case's ``input.dat`` (the native input layout) and ``--initial``
path, runs the solver with ``Running_steps`` = 1, 2, 5, 6, 100, 101, 199 and
200 (each run from the same initial path, so consecutive counts give single
iterations at several points of the run), and keeps its
path files (``<out>.initial`` / ``<out>.final``: seven ``%.17g`` columns a b c
alpha beta gamma E, RC_main.cu:2555-2585) and its stdout summary lines
(``info:``, ``legacy_selection:``, ``final_convergence:``, ``path_review:``).
Back on any machine,

    python tests/golden/make_string_golden.py collect --from <dir>

packs them with the case arrays into ``string_reference.npz`` beside this
script.  The solver runs with STRING_DISABLE_LONG_COUL=1 (RC_main.cu:478):
every site is neutral, so the long-range Coulomb grid is zero anyway.

Cases (seeded, from ``string_vext_b200.synth``):

* ``c4``   -- the String-path workload: the 64-atom small_field framework,
  64 images along the fractional c axis at (0.25, 0.25), random unit
  quaternions (seed 3) as Euler angles in [0, 2 pi); direction 3.
* ``skew`` -- the first batch framework (seed 4) with at most 300 atoms and
  the first guest (98 K, 3.75 A, 1.54 A): 45 images along a at
  (b, c) = (0.3, 0.6), random quaternions (seed 11); direction 1.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
SOLVER = REPO / "oracle" / "_ref" / "string_triclinic_cuda"
STEPS = (1, 2, 5, 6, 100, 101, 199, 200)
DELTA_FRAC = 1e-4
DELTA_ANGLE_DEG = 1.0
MARKERS = ("info:", "legacy_selection:", "final_convergence:", "path_review:")


def cases():
    sys.path.insert(0, str(REPO))
    from string_vext_b200 import synth
    from string_vext_b200.string_path import euler_from_quaternions

    out = {}
    case, frac, quat, _, _ = synth.string_path()
    out["c4"] = (case, np.column_stack([frac, np.mod(euler_from_quaternions(quat), 2 * np.pi)]), 3)
    framework = next(c for c in synth.batch_frameworks()[::2] if len(c["frame_frac"]) <= 300)
    n = 45
    rng = np.random.default_rng(11)
    frac = np.column_stack([np.linspace(0.0, 1.0, n), np.full(n, 0.3), np.full(n, 0.6)])
    euler = np.mod(euler_from_quaternions(synth.random_quaternions(rng, n)), 2 * np.pi)
    out["skew"] = (framework, np.column_stack([frac, euler]), 1)
    return out


def run(out_dir: Path) -> None:
    from string_vext_b200.input import write_string_input

    if not SOLVER.exists():
        raise SystemExit(f"{SOLVER} missing: make -C oracle string REF=<reference checkout>")
    env = dict(os.environ, STRING_DISABLE_LONG_COUL="1", STRING_CUDA_DEVICE="0")
    for name, (case, path, direction) in cases().items():
        for steps in STEPS:
            work = out_dir / f"{name}_{steps}"
            work.mkdir(parents=True, exist_ok=True)
            write_string_input(case, work / "input.dat", n_points=len(path),
                               delta_frac=DELTA_FRAC, delta_angle_deg=DELTA_ANGLE_DEG,
                               direction=direction, running_steps=steps)
            (work / "initial.dat").write_text(
                "\n".join("\t".join(f"{v:.17g}" for v in row) for row in path) + "\n")
            proc = subprocess.run([str(SOLVER), "input.dat", "initial.dat", "path.dat"],
                                  cwd=work, env=env, capture_output=True, text=True,
                                  timeout=900)
            (work / "stdout.txt").write_text(proc.stdout)
            (work / "stderr.txt").write_text(proc.stderr)
            print(f"{name} steps={steps} rc={proc.returncode}", flush=True)
            if proc.returncode != 0:
                raise SystemExit(f"solver failed on {name}/{steps}: {proc.stderr[-400:]}")


def collect(src: Path) -> None:
    arrays = {}
    meta = {}
    for name, (case, path, direction) in cases().items():
        arrays[f"{name}_cell"] = case["cell"]
        arrays[f"{name}_frac"] = case["frame_frac"]
        arrays[f"{name}_sigma"] = case["frame_sigma"]
        arrays[f"{name}_epsilon"] = case["frame_epsilon"]
        arrays[f"{name}_guest"] = np.array([case["guest_epsilon"][0], case["guest_sigma"][0],
                                            case["bond_length"], case["cutoff"],
                                            case["temperature"], case["total_mass"]])
        arrays[f"{name}_lengths_angles"] = np.array(list(case["cell_lengths"])
                                                    + list(case["cell_angles_deg"]))
        arrays[f"{name}_start"] = path
        meta[name] = {"direction": direction, "delta_frac": DELTA_FRAC,
                      "delta_angle_deg": DELTA_ANGLE_DEG, "steps": list(STEPS)}
        for steps in STEPS:
            work = src / f"{name}_{steps}"
            initial = np.loadtxt(work / "path.dat.initial")
            final = np.loadtxt(work / "path.dat.final")
            if steps == STEPS[0]:
                arrays[f"{name}_initial"] = initial
            else:
                assert np.array_equal(initial, arrays[f"{name}_initial"])
            arrays[f"{name}_final_{steps}"] = final
            lines = [ln.strip() for ln in (work / "stdout.txt").read_text().split("\n")]
            found = []
            for ln in lines:
                for marker in MARKERS:
                    at = ln.find(marker)
                    if at >= 0:
                        found.append(ln[at:])
            meta[name][f"stdout_{steps}"] = found
    arrays["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(HERE / "string_reference.npz", **arrays)
    print("wrote", HERE / "string_reference.npz")


def main():
    parser = argparse.ArgumentParser(description=__doc__,
                                     formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = parser.add_subparsers(dest="cmd", required=True)
    p_run = sub.add_parser("run")
    p_run.add_argument("--out", type=Path, required=True)
    p_col = sub.add_parser("collect")
    p_col.add_argument("--from", dest="src", type=Path, required=True)
    args = parser.parse_args()
    sys.path.insert(0, str(REPO))
    if args.cmd == "run":
        run(args.out)
    else:
        collect(args.src)


if __name__ == "__main__":
    main()
