"""Vext field kernels through the C ABI against the FP64 oracle and the
reference's golden outputs.

Tolerances (the stated bar): the FP64 kernel agrees with the oracle to 1e-10
relative (floor 1 K); the mixed-precision kernel agrees with the FP64 kernel
to 1e-4 K absolute where E <= 0 and 1e-6 relative (floor 1 K) where E > 0.
"""
import numpy as np
import pytest

from oracle import oracle
from string_vext_b200 import _lib, synth
from string_vext_b200.orientation import normalized_directors, regular_pose_grid
from string_vext_b200.system import VextSystem
from string_vext_b200.vext import calculate_vext

pytestmark = pytest.mark.gpu

FP64 = _lib.VEXT_MODE_FP64
MIXED = _lib.VEXT_MODE_MIXED


def rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1.0)


def assert_mixed_ok(mixed, exact):
    neg = exact <= 0
    if neg.any():
        assert np.abs(mixed - exact)[neg].max() < 1e-4
    if (~neg).any():
        assert rel(mixed, exact)[~neg].max() < 1e-6


def grid(size, n_axes=64):
    centers, axes = regular_pose_grid(size, n_axes)
    return centers, normalized_directors(axes)


@pytest.mark.parametrize("maker,size", [(synth.small_field, 4), (synth.full_field, 3),
                                        (synth.skewed_field, 3)])
@pytest.mark.parametrize("cb", [16, 32])
def test_fp64_and_mixed_match_oracle(maker, size, cb):
    case = maker()
    centers, axes = grid(size)
    ref = oracle.pose_energy(case, centers, axes)
    with VextSystem(case) as system:
        e64 = system.field(size, axes, mode=FP64, energy=True, centers_per_region=cb)["energy"]
        plain = system.field(size, axes, mode=_lib.VEXT_MODE_FP64_PLAIN, energy=True,
                             centers_per_region=cb)["energy"]
        mixed = system.field(size, axes, mode=MIXED, energy=True, centers_per_region=cb)
    assert rel(e64, ref).max() < 1e-10
    assert rel(plain, ref).max() < 1e-10
    assert_mixed_ok(mixed["energy"], ref)
    np.testing.assert_array_equal(mixed["orientation_K"],
                                  mixed["energy"].T.reshape(64, size, size, size).astype(np.float32))


def test_calculate_vext_channels_against_reference_golden(golden):
    g = golden("small_field_s4.npz")
    case = synth.small_field()
    out, stats = calculate_vext(case, size=4, orientations=64, mode=FP64, return_stats=True)
    # float32 storage of FP64 values that agree to ~1e-13: equal or 1 ulp apart
    np.testing.assert_allclose(out["orientation_K"], g["orientation_K"], rtol=2.4e-7, atol=0)
    np.testing.assert_allclose(out["marginal_K"], g["marginal_K"], rtol=2.4e-7, atol=1e-6)
    np.testing.assert_allclose(out["site_K"], g["site_K"], rtol=2.4e-7, atol=1e-6)
    np.testing.assert_allclose(out["grid"], g["grid"], rtol=2.4e-7, atol=1e-7)
    assert stats["poses"] == 4 ** 3 * 64
    mixed = calculate_vext(case, size=4, orientations=64)
    np.testing.assert_allclose(mixed["orientation_K"], g["orientation_K"], rtol=1e-6, atol=1e-4)


def test_toy_skew_cell(golden, tmp_path):
    from string_vext_b200.input import parse_string_input
    g = golden("toy_skew.npz")
    path = tmp_path / "input.dat"
    path.write_text(str(g["toy_input"]))
    case = parse_string_input(path)
    out = calculate_vext(case, size=3, orientations=4)
    # the reference unit test's own comparison (tests/unit/test_public_api.py:60-61)
    np.testing.assert_allclose(out["orientation_K"].reshape(4, -1).T, g["toy_direct"],
                               rtol=1e-6, atol=1e-3)
    assert out["site_K"].shape == (2, 3, 3, 3)


def test_cli_writes_npz_and_provenance_exclusively(golden, tmp_path):
    """The CLI contract of the reference (src/string_vext/vext.py:46-84): an
    NPZ of the output channels plus a provenance JSON beside it, neither ever
    overwritten."""
    import json

    from string_vext_b200 import vext
    g = golden("toy_skew.npz")
    inp = tmp_path / "input.dat"
    inp.write_text(str(g["toy_input"]))
    out = tmp_path / "fields" / "toy.npz"
    vext.main(["--input", str(inp), "--output", str(out), "--size", "3",
               "--orientations", "4"])
    with np.load(out) as f:
        assert set(f.files) == {"orientation_K", "marginal_K", "site_K", "axes", "cell_matrix",
                                "atom_fractional", "framework_sigma_A", "framework_epsilon_K",
                                "grid"}
        np.testing.assert_allclose(f["orientation_K"].reshape(4, -1).T, g["toy_direct"],
                                   rtol=1e-6, atol=1e-3)
    record = json.loads(out.with_suffix(".json").read_text())
    assert record["size"] == 3 and record["orientations"] == 4
    assert len(record["output_sha256"]) == 64 and len(record["kernel_sha256"]) == 64
    assert sorted(p.name for p in out.parent.iterdir()) == ["toy.json", "toy.npz"]
    before = out.read_bytes()
    with pytest.raises(FileExistsError):
        vext.main(["--input", str(inp), "--output", str(out), "--size", "3",
                   "--orientations", "4"])
    assert out.read_bytes() == before


@pytest.mark.parametrize("size,n_axes", [(1, 4), (5, 5), (7, 64), (9, 130)])
def test_ragged_sizes(size, n_axes):
    case = synth.small_field()
    centers, axes = grid(max(size, 2), n_axes)
    if size == 1:
        centers = np.full((1, 3), 0.5)
    ref = oracle.pose_energy(case, centers, axes)
    with VextSystem(case) as system:
        e = system.field(size, axes, mode=MIXED, energy=True)["energy"]
    assert_mixed_ok(e, ref)


def test_full_size_field_properties():
    """60^3 x 64 on the full-size workload: mixed vs FP64 kernel (the bench's
    error statement), marginal/site/grid finite, float32 channel = cast."""
    case = synth.full_field()
    _, axes = grid(60)
    with VextSystem(case) as system:
        exact = system.field(60, axes, mode=FP64, energy=True, orientation=False)["energy"]
        mixed = system.field(60, axes, mode=MIXED, energy=True, marginal=True, site=True,
                             grid=True)
        stats = system.last_stats
    assert_mixed_ok(mixed["energy"], exact)
    assert stats["poses"] == 60 ** 3 * 64
    assert np.isfinite(mixed["marginal_K"]).all() and np.isfinite(mixed["site_K"]).all()
    np.testing.assert_array_equal(mixed["site_K"][0], mixed["site_K"][1])
    # marginal from the device epilogue vs host logsumexp of the same energies
    from string_vext_b200.physics import marginal_energy
    host = marginal_energy(mixed["energy"], case["temperature"]).astype(np.float32)
    np.testing.assert_allclose(mixed["marginal_K"].reshape(-1), host, rtol=1e-6, atol=1e-4)


def test_periodicity_of_the_field():
    """Shifting every center by a whole lattice vector changes nothing: the
    fields of two grids that are the same points mod 1 agree."""
    case = synth.skewed_field()
    centers, axes = grid(4)
    with VextSystem(case) as system:
        e1, *_ = system.pose_energy_grad(centers @ case["cell"],
                                         np.tile([1.0, 0, 0, 0], (len(centers), 1)),
                                         mode=FP64, grad=False)
        e2, *_ = system.pose_energy_grad((centers + [3, -2, 1]) @ case["cell"],
                                         np.tile([1.0, 0, 0, 0], (len(centers), 1)),
                                         mode=FP64, grad=False)
    np.testing.assert_allclose(e1, e2, rtol=1e-10, atol=1e-8)


def test_fp32_naive_mode_is_bounded_and_worse_than_mixed():
    """The precision study's naive FP32 field (plain loop, FP32 sum) stays
    within FP32 rounding of the oracle, and the mixed field is more accurate."""
    case = synth.small_field()
    centers, axes = grid(4)
    ref = oracle.pose_energy(case, centers, axes)
    with VextSystem(case) as system:
        naive = system.field(4, axes, mode=_lib.VEXT_MODE_FP32_NAIVE, energy=True,
                             orientation=False)["energy"]
        mixed = system.field(4, axes, energy=True, orientation=False)["energy"]
    assert np.isfinite(naive).all()
    err_naive = np.abs(naive - ref) / np.maximum(np.abs(ref), 1.0)
    err_mixed = np.abs(mixed - ref) / np.maximum(np.abs(ref), 1.0)
    assert err_naive.max() < 1e-3
    assert err_mixed.max() < 0.1 * err_naive.max()


def test_off_center_sites_forward_field():
    """Unequal site masses put the sites off-center (o_1 != -o_0): the
    forward field (FP64 and mixed) against the oracle on small_field and the
    skewed workload."""
    for maker in (synth.small_field, synth.skewed_field):
        case = dict(maker())
        case["guest_mass"] = np.array([15.0, 25.0])
        case["total_mass"] = 40.0
        centers, axes = grid(4)
        ref = oracle.pose_energy(case, centers, axes)
        with VextSystem(case) as system:
            e64 = system.field(4, axes, mode=FP64, energy=True)["energy"]
            mixed = system.field(4, axes, mode=MIXED, energy=True)["energy"]
        assert rel(e64, ref).max() < 1e-10
        assert_mixed_ok(mixed, ref)


def test_list_classes_cover_the_outer_shell():
    """Every region's shell ends with its outer entries (beyond rc + the region
    radius of the origin, where at most one site of a director is inside the
    cutoff and the batched kernels evaluate that site alone).  On full_field
    they are a sizeable part of the list, they lie beyond the near class, and
    the per-field path (which evaluates both sites there) still matches the
    FP64 oracle on a sample of poses whose pairs reach into them."""
    case = synth.full_field()
    size = 6
    centers, axes = regular_pose_grid(size, 64)
    axes = normalized_directors(axes)
    with VextSystem(case) as system:
        out = system.field(size, axes, energy=True, orientation=False)
        st = system.last_stats
    assert 0 < st["outer_entries"] < st["list_entries"] - st["near_entries"]
    # the outer shell of a 16-center region: rc + rho + 1e-3 A to rc + max|o| + rho,
    # about a tenth of the list
    assert 0.05 < st["outer_entries"] / st["list_entries"] < 0.3
    pick = np.arange(0, len(centers), 37)
    assert_mixed_ok(out["energy"][pick], oracle.pose_energy(case, centers[pick], axes))
