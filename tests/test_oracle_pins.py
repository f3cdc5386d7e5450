"""Pin the FP64 oracle against the reference's own outputs (golden fixtures
made by tests/golden/make_golden.py from the reference code) and its
known-answer tests.  CPU only."""
import numpy as np
import pytest

from conftest import case_from_golden
from oracle import oracle
from string_vext_b200 import synth
from string_vext_b200.input import parse_string_input
from string_vext_b200.orientation import regular_pose_grid
from string_vext_b200.physics import marginal_energy


def rel_err(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1.0)


def test_toy_skew_cell_direct(golden, tmp_path):
    g = golden("toy_skew.npz")
    path = tmp_path / "input.dat"
    path.write_text(str(g["toy_input"]))
    case = parse_string_input(path)
    centers, axes = regular_pose_grid(3, 4)
    axes = axes / np.linalg.norm(axes, axis=1, keepdims=True)
    energy = oracle.pose_energy(case, centers, axes)
    assert rel_err(energy, g["toy_direct"]).max() < 1e-10
    # the reference unit test's own tolerance for its stored float32 field
    np.testing.assert_allclose(g["toy_orientation_K"].reshape(4, -1).T, energy,
                               rtol=1e-6, atol=1e-3)


def test_small_field_direct_native_and_channels(golden):
    g = golden("small_field_s4.npz")
    case = case_from_golden(g)
    np.testing.assert_array_equal(case["cell"], synth.small_field()["cell"])
    energy = oracle.pose_energy(case, g["centers"], g["axes"])
    assert rel_err(energy, g["direct"]).max() < 1e-10
    assert rel_err(energy, g["native"]).max() < 1e-10
    # float32 channels of calculate_vext
    np.testing.assert_allclose(energy.T.reshape(64, 4, 4, 4), g["orientation_K"], rtol=2e-7)
    marginal = marginal_energy(g["native"], case["temperature"]).astype(np.float32)
    np.testing.assert_array_equal(marginal.reshape(4, 4, 4), g["marginal_K"])
    site = oracle.site_energy(case, g["centers"] @ case["cell"])
    np.testing.assert_allclose(np.stack([site, site]).reshape(2, 4, 4, 4), g["site_K"], rtol=2e-7)


@pytest.mark.parametrize("name,maker", [("full_field", synth.full_field),
                                        ("skewed_field", synth.skewed_field)])
def test_sampled_centers_of_large_workloads(golden, name, maker):
    g = golden(f"{name}_sample.npz")
    case = maker()
    energy = oracle.pose_energy(case, g["centers"], g["axes"])
    assert rel_err(energy, g["direct"]).max() < 1e-10
    assert rel_err(energy, g["native"]).max() < 1e-10


def test_csr_kernel_restatement_is_bit_exact(golden):
    g = golden("csr_batch.npz")
    case = synth.small_field()
    drv = oracle.ReferenceDriver(case, oracle.LIB_PATH, symbol="oracle_reused_neighbors")
    assert len(drv.images) == int(g["n_images"])
    out = np.zeros_like(g["output"])
    code = drv.kernel(len(g["centers"]), 64, len(drv.images), float(g["cutoff2"]),
                      *(oracle._ptr(np.ascontiguousarray(a)) for a in (
                          g["centers"], g["axes"], drv.images, g["offsets"], drv.coeff12,
                          drv.coeff6, drv.shift, drv.floor2, g["starts"], g["indices"], out)))
    assert code == 0
    np.testing.assert_array_equal(out, g["output"])


def test_pair_function_known_answers(golden):
    g = golden("pair_lj.npz")
    ours = np.array([oracle.pair_lj(c, s, a, cutoff=rc) for c, s, a, rc in
                     zip(g["cells"], g["sites"], g["atoms"], g["cutoffs"])])
    np.testing.assert_allclose(ours, g["energy"], rtol=1e-12, atol=1e-9)
    # the reference test's assertions (test_native_string_triclinic.py:59-90)
    np.testing.assert_allclose(ours, g["brute"], rtol=2e-10, atol=1e-6)
    assert ours[0] > 1e6                       # skew counterexample needs the far image
    assert np.isfinite(ours[-2]) and ours[-2] > 1e12   # contact floor
    assert abs(ours[-1]) < 1e-10               # exactly zero at the cutoff
    periodic = ours[-8:-2]                     # same pair under lattice shifts
    np.testing.assert_allclose(periodic, periodic[0], rtol=1e-10, atol=1e-7)


def test_euler_pose_energy(golden):
    g = golden("euler_poses.npz")
    energy = oracle.euler_pose_energy(synth.small_field(), g["poses"])
    np.testing.assert_allclose(energy, g["energy"], rtol=1e-12, atol=1e-9)


def test_oracle_gradient_matches_central_differences():
    case = synth.small_field()
    rng = np.random.default_rng(5)
    centers = rng.random((6, 3)) @ case["cell"]
    u = rng.normal(size=(6, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    e, gc, gu = oracle.pose_energy_grad(case, centers, u)
    h = 1e-5
    for k in range(3):
        d = np.zeros(3)
        d[k] = h
        ep, _, _ = oracle.pose_energy_grad(case, centers + d, u)
        em, _, _ = oracle.pose_energy_grad(case, centers - d, u)
        np.testing.assert_allclose((ep - em) / (2 * h), gc[:, k], rtol=1e-5,
                                   atol=1e-5 * np.abs(gc).max())
        ep, _, _ = oracle.pose_energy_grad(case, centers, u + d)
        em, _, _ = oracle.pose_energy_grad(case, centers, u - d)
        np.testing.assert_allclose((ep - em) / (2 * h), gu[:, k], rtol=1e-5,
                                   atol=1e-5 * np.abs(gu).max())


def test_pair_counts_small_field():
    case = synth.small_field()
    centers, axes = regular_pose_grid(4, 64)
    counts = oracle.pair_counts(case, centers, axes / np.linalg.norm(axes, axis=1, keepdims=True))
    assert 450 < counts.mean() < 500            # ~475 in-cutoff pairs per pose
