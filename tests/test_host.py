"""Host logic and the C-ABI boundary without a GPU: the library loads, exports
every symbol include/vext_b200.h declares, rejects bad arguments the way the
reference does before touching the device; input/grid/cell mirrors; the
seeded workload generator."""
import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT
from string_vext_b200 import _lib, synth
from string_vext_b200.cell import cell_matrix
from string_vext_b200.input import parse_string_input, write_string_input
from string_vext_b200.orientation import regular_pose_grid


def declared_symbols():
    text = (ROOT / "include" / "vext_b200.h").read_text()
    return sorted(set(re.findall(r"VEXT_API\s+[\w\s\*]+?\b(\w+)\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert "evaluate_reused_neighbors" in names and len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert _lib.version().startswith("vext_b200")


def dropin(n_centers, n_axes, n_images, cutoff2, starts, indices):
    lib = _lib.load()
    z = np.zeros(64)
    out = np.zeros(64)
    s = np.ascontiguousarray(starts, dtype=np.int64)
    i = np.ascontiguousarray(indices, dtype=np.int32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    return lib.evaluate_reused_neighbors(n_centers, n_axes, n_images, cutoff2, p(z), p(z), p(z),
                                         p(z), p(z), p(z), p(z), p(z), p(s), p(i), p(out))


def test_dropin_codes_before_device_work():
    # code 1 (kernel.cpp:11-12)
    assert dropin(-1, 4, 1, 1.0, [0, 0], [0]) == 1
    assert dropin(1, 0, 1, 1.0, [0, 0], [0]) == 1
    assert dropin(1, 4, 0, 1.0, [0, 0], [0]) == 1
    assert dropin(1, 4, 1, 0.0, [0, 0], [0]) == 1
    assert dropin(0, 4, 1, 1.0, [0], [0]) == 0          # nothing to do
    # code 2 / 3 at the first center: returned before any CUDA call
    assert dropin(1, 4, 1, 1.0, [1, 0], [0]) == 2
    assert dropin(1, 4, 2, 1.0, [0, 2], [0, 2]) == 3
    assert dropin(1, 4, 2, 1.0, [0, 1], [-1]) == 3
    assert dropin(1, 4, 2, 1.0, [-1, 1], [0, 0]) == 2    # negative start (extension)


def test_cell_matrix_matches_reference_formula():
    m = cell_matrix([12.0, 13.0, 14.0], [90.0, 115.152, 90.0])
    assert m[2, 0] < 0 and abs(np.linalg.norm(m[2]) - 14.0) < 1e-12
    with pytest.raises(ValueError):
        cell_matrix([1, 1, 1], [90, 90, 180])
    with pytest.raises(ValueError):
        cell_matrix([1, 1, 1], [10, 10, 170])


def test_input_roundtrip(golden, tmp_path):
    g = golden("toy_skew.npz")
    path = tmp_path / "input.dat"
    path.write_text(str(g["toy_input"]))
    case = parse_string_input(path)
    assert case["cell"][2, 0] < 0
    assert abs(np.linalg.norm(case["cell"][2]) - 14.0) < 1e-12
    np.testing.assert_allclose(case["guest_xyz"][:, 0], [-0.77, 0.77])
    out = tmp_path / "again.dat"
    write_string_input(case, out)
    again = parse_string_input(out)
    for key in ("cell", "frame_frac", "frame_sigma", "frame_epsilon", "guest_xyz"):
        np.testing.assert_allclose(again[key], case[key], rtol=1e-15, atol=1e-15)


def test_grid_layout():
    centers, axes = regular_pose_grid(3, 4)
    assert centers.shape == (27, 3) and axes.shape == (4, 3)
    np.testing.assert_array_equal(centers[1], [1 / 6, 1 / 6, 0.5])   # k fastest
    np.testing.assert_allclose(np.linalg.norm(axes, axis=1), 1.0)


def test_synthetic_workloads_are_deterministic():
    a, b = synth.full_field(), synth.full_field()
    np.testing.assert_array_equal(a["frame_frac"], b["frame_frac"])
    assert len(a["frame_frac"]) == 600 and a["cutoff"] == 12.8
    assert len(synth.skewed_field()["frame_frac"]) == 3000
    cases = synth.batch_frameworks(5)
    assert len(cases) == 10
    for c in cases:
        assert 100 <= len(c["frame_frac"]) <= 4000
    case, pf, pq, bf, bq = synth.string_path()
    assert pf.shape == (64, 3) and bq.shape == (65536, 4)
    np.testing.assert_allclose(np.linalg.norm(pq, axis=1), 1.0)
