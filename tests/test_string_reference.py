"""The String iteration of oracle/string_oracle.py pinned to the reference
String solver's own output.

tests/golden/string_reference.npz holds path files written by the
reference's String program (native/string/source_code/RC_main.cu, built
unchanged from source and run with ``--initial`` on a GPU; generated by
tests/golden/make_string_golden.py) after 1, 2, 5, 6, 100, 101, 199 and 200
iterations, for the String-path workload (64 images along c, direction 3)
and a skewed framework (45 images along a, direction 1).  Every run starts
from the same initial path, so consecutive counts give single iterations
early, in the middle and at the end of a 200-iteration run.

Checked here:
* the energy column of every stored path against the oracle's FP64 energy of
  that path (1e-12 relative, floor 1e-8 K);
* the restated iteration with the reference's one-sided-difference forces,
  from the initial path for 1, 2, 5 and 6 iterations and as single
  iterations k -> k + 1 from the reference's own path after k iterations:
  positions to 1e-10 (fractional), angles to 1e-9 rad.  The reference's
  forces are differences E(x + h) - E(x) of FP64 energies that it sums in
  another order, so an image whose energy dwarfs its forces (a site on top
  of an atom: image 53 of the String-path workload sits at 3e14 K) carries a
  step-direction uncertainty of about 256 eps |E| / |force|; that allowance
  is added (per image for angles; for positions the largest one, which the
  reparametrisation passes along the path);
* the end-of-run summary lines (convergence flags, log-domain scores, the
  chosen stage, peak energies) against the solver's stdout.

Longer runs are not compared path for path: after many iterations two FP64
implementations that sum energies in different orders take different
discrete branches (an angle step kept or rejected on E2 > E0, at ties within
FP64 rounding), so the paths part by whole steps while each iteration stays
the reference's -- which the single-iteration checks at 100 and 199 show.
"""
import json
import re

import numpy as np
import pytest

from oracle import oracle, string_oracle
from string_vext_b200 import synth, tst

PI = 3.141592653589793
EPS = np.finfo(float).eps


def load_case(g, name):
    lengths_angles = g[f"{name}_lengths_angles"]
    eps, sig, bond, cutoff, temperature, _ = g[f"{name}_guest"]
    case = synth.make_case(lengths_angles[:3], lengths_angles[3:], g[f"{name}_frac"],
                           g[f"{name}_sigma"], g[f"{name}_epsilon"], (eps, sig, bond), cutoff,
                           temperature)
    np.testing.assert_array_equal(case["cell"], g[f"{name}_cell"])
    return case


def fields(line):
    return dict(re.findall(r"(\w+)=(\S+)", line))


def step_tolerances(case, path, hf, ha, steps=1):
    """Allowances (positions, angles) for `steps` iterations from `path`:
    1e-10 / 1e-9 plus the step-direction uncertainty of forces that are
    differences of FP64 energies of magnitude |E|.  Angles per image, plus
    the smoothing's share (coefficient 1e-4) of the neighbours' allowance;
    the positions of every image take the largest allowance, because the
    equal-arc-length reparametrisation passes one image's position on to
    the images after it."""
    grad = oracle.string_fd_gradient(case, path, delta_frac=hf, delta_angle_rad=ha)
    energy = np.abs(string_oracle.pose_energy(case, path))
    unc = 256 * EPS * np.maximum(energy, 1.0)
    gt = np.maximum(np.linalg.norm(grad[:, :3], axis=1), unc)
    gr = np.maximum(np.linalg.norm(grad[:, 3:], axis=1), unc)
    ang = steps * 4 * ha * unc / gr
    near = np.maximum(np.r_[0.0, ang[:-1]], np.r_[ang[1:], 0.0])
    return (1e-10 + steps * 4 * hf * (unc / gt).max()), (1e-9 + ang + 1e-4 * near)[:, None]


def assert_path_close(got, ref, tol_pos, tol_ang, what):
    dp = np.abs(got[:, :3] - ref[:, :3])
    da = np.abs(got[:, 3:] - ref[:, 3:6])
    assert (dp <= tol_pos).all(), f"{what}: positions off by {dp.max():.3g}"
    assert (da <= tol_ang).all(), f"{what}: angles off by {da.max():.3g}"


@pytest.fixture(scope="module")
def reference(golden):
    g = golden("string_reference.npz")
    return g, json.loads(str(g["meta"]))


@pytest.mark.parametrize("name", ["c4", "skew"])
def test_energy_column_of_every_reference_path(reference, name):
    g, meta = reference
    case = load_case(g, name)
    for key in [f"{name}_initial"] + [f"{name}_final_{k}" for k in meta[name]["steps"]]:
        path = g[key]
        np.testing.assert_allclose(string_oracle.pose_energy(case, path[:, :6]), path[:, 6],
                                   rtol=1e-12, atol=1e-8, err_msg=key)


@pytest.mark.parametrize("name", ["c4", "skew"])
def test_iterations_from_the_initial_path(reference, name):
    g, meta = reference
    m = meta[name]
    case = load_case(g, name)
    hf, ha = m["delta_frac"], m["delta_angle_deg"] * PI / 180
    start = g[f"{name}_start"]
    np.testing.assert_array_equal(g[f"{name}_initial"][:, :6], start)
    s, done = start.copy(), 0
    for steps in [k for k in m["steps"] if k <= 6]:
        tol_pos, tol_ang = step_tolerances(case, start, hf, ha, steps)
        while done < steps:
            s, stop, _, _ = string_oracle.iteration(case, s, hf=hf, ha=ha,
                                                    direction=m["direction"], gradient="fd")
            assert not stop
            done += 1
        assert_path_close(s, g[f"{name}_final_{steps}"], tol_pos, tol_ang, f"{steps} iterations")


@pytest.mark.parametrize("name", ["c4", "skew"])
@pytest.mark.parametrize("k", [1, 5, 100, 199])
def test_single_iterations_along_the_run(reference, name, k):
    g, meta = reference
    m = meta[name]
    case = load_case(g, name)
    hf, ha = m["delta_frac"], m["delta_angle_deg"] * PI / 180
    before = g[f"{name}_final_{k}"][:, :6]
    s, stop, totals, _ = string_oracle.iteration(case, before, hf=hf, ha=ha,
                                                 direction=m["direction"], gradient="fd")
    assert not stop
    tol_pos, tol_ang = step_tolerances(case, before, hf, ha)
    assert_path_close(s, g[f"{name}_final_{k + 1}"], tol_pos, tol_ang, f"iteration {k} -> {k + 1}")
    if k + 1 == 200:
        # the convergence flags the solver prints after its last iteration
        conv = fields(next(ln for ln in m["stdout_200"] if ln.startswith("final_convergence:")))
        n = len(s)
        assert int(conv["coordinate_current"]) == int(totals[0] < 0.3 * hf * n * np.sqrt(3))
        assert int(conv["orientation_current"]) == int(totals[1] < 0.3 * ha * n * np.sqrt(3))


@pytest.mark.parametrize("name", ["c4", "skew"])
def test_end_of_run_summary(reference, name):
    """Scores of the initial and the final path, the chosen stage and the peak
    energies against the solver's stdout (RC_main.cu:2396-2553)."""
    g, meta = reference
    m = meta[name]
    case = load_case(g, name)
    T, mass = case["temperature"], case["total_mass"]
    hop = case["cell_lengths"][m["direction"] - 1]
    initial = g[f"{name}_initial"]
    for steps in m["steps"]:
        final = g[f"{name}_final_{steps}"]
        out = m[f"stdout_{steps}"]
        info = next(ln for ln in out if ln.startswith("info:")).split()
        assert int(info[2]) == steps and int(info[3]) == len(case["frame_frac"])
        sel = fields(next(ln for ln in out if ln.startswith("legacy_selection:")))
        ok_i, logd_i = tst.log_score(initial[:, :6], initial[:, 6], case["cell"], T, mass, hop)
        ok_f, logd_f = tst.log_score(final[:, :6], final[:, 6], case["cell"], T, mass, hop)
        assert ok_i and ok_f
        np.testing.assert_allclose([logd_i, logd_f],
                                   [float(sel["logD_initial"]), float(sel["logD_final"])],
                                   rtol=1e-12)
        chosen = "initial" if tst.choose_initial((ok_i, logd_i), (ok_f, logd_f)) else "final"
        assert chosen == sel["chosen_stage"]
        review = fields(next(ln for ln in out if ln.startswith("path_review:")))
        assert float(review["peak_initial_K"]) == initial[:, 6].max()
        assert float(review["peak_final_K"]) == final[:, 6].max()
