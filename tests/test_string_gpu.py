"""GPU String path update through the C ABI against a CPU restatement of the
reference iteration (oracle/string_oracle.py, global.h:1281-2244), with the
same analytic FP64 gradient; consistency with the reference's own
finite-difference forces; the path-file format."""
import numpy as np
import pytest

from oracle import string_oracle
from string_vext_b200 import _lib, synth
from string_vext_b200.string_path import (euler_from_quaternions, path_selection,
                                          quaternions_from_euler, read_initial, run_string,
                                          write_path)
from string_vext_b200.system import VextSystem

pytestmark = pytest.mark.gpu

FP64 = _lib.VEXT_MODE_FP64


def path_config4():
    case, frac, quat, _, _ = synth.string_path()
    euler = euler_from_quaternions(quat)
    euler = np.mod(euler, 2 * np.pi)
    return case, np.column_stack([frac, euler])


def test_euler_quaternion_roundtrip():
    rng = np.random.default_rng(0)
    q = rng.normal(size=(100, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    e = euler_from_quaternions(q)
    q2 = quaternions_from_euler(e)
    assert np.allclose(np.abs((q * q2).sum(1)), 1.0, atol=1e-12)


@pytest.mark.parametrize("n_iter", [1, 5])
def test_iterations_match_cpu_restatement(n_iter):
    case, s = path_config4()
    # direction 3: the path runs along c from (.25, .25, 0) to (.25, .25, 1)
    with VextSystem(case) as system:
        gpu, e_gpu, res = run_string(system, s, mode=FP64, direction=3, max_iterations=n_iter)
    ref = s.copy()
    for _ in range(n_iter):
        ref, stop, _, _ = string_oracle.iteration(case, ref, direction=3)
        assert not stop
    assert res["iterations"] == n_iter
    np.testing.assert_allclose(gpu[:, :3], ref[:, :3], rtol=0, atol=1e-10)
    np.testing.assert_allclose(gpu[:, 3:], ref[:, 3:], rtol=0, atol=1e-9)
    np.testing.assert_allclose(e_gpu, string_oracle.pose_energy(case, gpu), rtol=1e-10, atol=1e-8)


@pytest.mark.parametrize("n_images", [64, 45])
def test_end_fixing_matches_cpu_restatement(n_images):
    """Interior images pushed outside [0, 1] along the transport axis copy the
    nearest image inside (values before fixing); the ends keep their axis
    coordinate: one iteration against the CPU restatement, also for an image
    count that leaves a warp partly idle."""
    case, s = path_config4()
    s = s[np.linspace(0, len(s) - 1, n_images).round().astype(int)].copy()
    s[1:4, 2] = [-0.05, -0.03, -0.01]
    s[-4:-1, 2] = [1.01, 1.03, 1.05]
    with VextSystem(case) as system:
        gpu, _, res = run_string(system, s, mode=FP64, direction=3, max_iterations=1)
    ref, _, _, _ = string_oracle.iteration(case, s.copy(), direction=3)
    assert res["iterations"] == 1
    np.testing.assert_allclose(gpu[:, :3], ref[:, :3], rtol=0, atol=1e-10)
    np.testing.assert_allclose(gpu[:, 3:], ref[:, 3:], rtol=0, atol=1e-9)


def test_analytic_step_agrees_with_reference_fd_forces():
    """One step with the reference's one-sided forces (h = 1e-4 frac, 1 deg)
    versus the analytic forces: the positions move alike."""
    case, s = path_config4()
    fd, _, _, _ = string_oracle.iteration(case, s, direction=3, gradient="fd")
    with VextSystem(case) as system:
        gpu, _, _ = run_string(system, s, mode=FP64, direction=3, max_iterations=1)
    move_fd = fd[:, :3] - s[:, :3]
    move_gpu = gpu[:, :3] - s[:, :3]
    scale = np.abs(move_fd).max()
    assert scale > 0
    assert np.abs(move_gpu - move_fd).max() < 0.05 * scale


def test_string_run_200_iterations_and_files(tmp_path):
    case, s = path_config4()
    with VextSystem(case) as system:
        path, energy, res = run_string(system, s, direction=3, max_iterations=200)
    assert res["iterations"] == 200
    assert np.isfinite(path).all() and np.isfinite(energy).all()
    assert path[0, 2] == s[0, 2] and path[-1, 2] == s[-1, 2]   # ends fixed along c
    out = tmp_path / "string_path.dat"
    write_path(out, path, energy)
    lines = out.read_text().splitlines()
    assert len(lines) == 64 and all(len(ln.split()) == 7 for ln in lines)
    back = np.loadtxt(out)
    np.testing.assert_array_equal(back[:, :6], path)
    np.testing.assert_array_equal(back[:, 6], energy)
    # end-of-run summary: diffusivity and the initial / final path choice
    e0 = string_oracle.pose_energy(case, s)
    summary = path_selection(case, s, e0, path, energy, direction=3)
    assert summary["chosen"] in ("initial", "final")
    assert summary["diffusivity_final_m2_s"] >= 0
    init = tmp_path / "initial.dat"
    init.write_text("\n".join("\t".join(f"{v:.17g}" for v in row) for row in path) + "\n")
    np.testing.assert_array_equal(read_initial(init, 64), path)


@pytest.mark.parametrize("name", ["c4", "skew"])
def test_reference_difference_mode_reproduces_reference_solver(golden, name):
    """The GPU update with the reference's own one-sided-difference forces
    (VEXT_STRING_REFERENCE_FD, FP64 energies) against the path files of the
    reference String solver built from source: 1, 2, 5 and 6 iterations from
    the initial path, and single iterations from the reference's own path
    after 1, 5, 100 and 199 iterations; positions to 1e-10, angles to 1e-9 rad
    (plus, per image, the step-direction uncertainty of forces that are
    differences of FP64 energies, test_string_reference.step_tolerances);
    energies of the final paths to 1e-10 relative."""
    import json

    from test_string_reference import assert_path_close, load_case, step_tolerances
    g = golden("string_reference.npz")
    m = json.loads(str(g["meta"]))[name]
    case = load_case(g, name)
    hf, ha = m["delta_frac"], m["delta_angle_deg"] * np.pi / 180
    start = g[f"{name}_start"]
    runs = [(start, k, f"{name}_final_{k}") for k in m["steps"] if k <= 6]
    runs += [(g[f"{name}_final_{k}"][:, :6], 1, f"{name}_final_{k + 1}")
             for k in (1, 5, 100, 199)]
    with VextSystem(case) as system:
        for path0, steps, key in runs:
            path, energy, res = run_string(
                system, path0, mode=FP64, direction=m["direction"], max_iterations=steps,
                delta_frac=hf, delta_angle_rad=ha, gradient=_lib.VEXT_STRING_REFERENCE_FD)
            assert res["iterations"] == steps
            tol_pos, tol_ang = step_tolerances(case, path0, hf, ha, steps)
            assert_path_close(path, g[key], tol_pos, tol_ang, key)
            np.testing.assert_allclose(energy, string_oracle.pose_energy(case, path),
                                       rtol=1e-10, atol=1e-8)
