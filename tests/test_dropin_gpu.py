"""The drop-in ``evaluate_reused_neighbors`` through the C ABI: bit-identical
to the reference kernel (golden outputs of native/vext/kernel.cpp built from
source), the reference's error codes and partial-output behaviour."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from string_vext_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def call(lib, centers, axes, images, offsets, c12, c6, shift, floor2, starts, indices, cutoff2,
         n_centers=None, n_images=None):
    out = np.full((len(centers), len(axes)), -7.0)
    arrays = [np.ascontiguousarray(a) for a in (centers, axes, images, offsets, c12, c6, shift,
                                                 floor2)]
    s = np.ascontiguousarray(starts, dtype=np.int64)
    i = np.ascontiguousarray(indices, dtype=np.int32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    code = lib.evaluate_reused_neighbors(
        len(centers) if n_centers is None else n_centers, len(axes),
        len(images) if n_images is None else n_images, cutoff2,
        *(p(a) for a in arrays), p(s), p(i), p(out))
    return code, out


def driver(case):
    """The reference CPU driver restated by the oracle (images, per-image
    coefficients, kd-tree CSR batches) bound to this library."""
    return oracle.ReferenceDriver(case, _lib.LIB_PATH)


@pytest.fixture(scope="module")
def batch(golden):
    g = golden("csr_batch.npz")
    pot = driver(synth.small_field())
    assert len(pot.images) == int(g["n_images"])
    return g, pot


def test_csr_batch_bit_exact(batch):
    g, pot = batch
    code, out = call(_lib.load(), g["centers"], g["axes"], pot.images, g["offsets"], pot.coeff12,
                     pot.coeff6, pot.shift, pot.floor2, g["starts"], g["indices"],
                     float(g["cutoff2"]))
    assert code == 0
    np.testing.assert_array_equal(out, g["output"])


def test_driver_bit_exact_against_reference_native(golden):
    g = golden("small_field_s4.npz")
    ours = driver(synth.small_field()).evaluate(g["centers"], g["axes"])
    np.testing.assert_array_equal(ours, g["native"])
    for name, maker in (("full_field", synth.full_field), ("skewed_field", synth.skewed_field)):
        s = golden(f"{name}_sample.npz")
        ours = driver(maker()).evaluate(s["centers"], s["axes"])
        np.testing.assert_array_equal(ours, s["native"])


def test_same_results_as_reference_kernel_build(batch):
    """The restated reference kernel (oracle C, no contraction) on the same
    arguments gives the same bits; also after the caller mutates the cached
    coefficient arrays in place."""
    g, pot = batch
    lib = _lib.load()
    olib = oracle.load()
    c12 = pot.coeff12.copy()
    for scale in (1.0, 1.5):
        c12[:] = pot.coeff12 * scale
        args = (g["centers"], g["axes"], pot.images, g["offsets"], c12, pot.coeff6, pot.shift,
                pot.floor2, g["starts"], g["indices"], float(g["cutoff2"]))
        code, ours = call(lib, *args)
        ocode, ref = call(type("L", (), {"evaluate_reused_neighbors":
                                         olib.oracle_reused_neighbors})(), *args)
        assert code == ocode == 0
        np.testing.assert_array_equal(ours, ref)


def test_error_codes_and_partial_output(batch):
    g, pot = batch
    lib = _lib.load()
    starts = g["starts"].copy()
    base = (g["centers"][:3], g["axes"], pot.images, g["offsets"], pot.coeff12, pot.coeff6,
            pot.shift, pot.floor2)
    # code 2 at center 1: center 0 written, the rest untouched
    s = starts[:4].copy()
    s[2] = s[1] - 1
    code, out = call(lib, *base, s, g["indices"], float(g["cutoff2"]))
    assert code == 2
    np.testing.assert_array_equal(out[0], g["output"][0])
    assert (out[1:] == -7.0).all()
    # code 3 at center 2
    idx = g["indices"].copy()
    idx[starts[2]] = len(pot.images)
    code, out = call(lib, *base, starts[:4], idx, float(g["cutoff2"]))
    assert code == 3
    np.testing.assert_array_equal(out[:2], g["output"][:2])
    # code 4: NaN coordinates on images listed for center 1 but not center 0
    images = pot.images.copy()
    only1 = sorted(set(g["indices"][starts[1]:starts[2]]) - set(g["indices"][:starts[1]]))
    assert only1
    images[only1] = np.nan
    code, out = call(lib, g["centers"][:3], g["axes"], images, g["offsets"], pot.coeff12,
                     pot.coeff6, pot.shift, pot.floor2, starts[:4], g["indices"],
                     float(g["cutoff2"]))
    assert code == 4
    np.testing.assert_array_equal(out[0], g["output"][0])
    assert (out[1] == -7.0).all()


def test_empty_neighbour_rows_and_odd_axis_counts(batch):
    g, pot = batch
    lib = _lib.load()
    centers = g["centers"][:5]
    starts = np.array([0, 0, 3, 3, 3, 10], dtype=np.int64)
    idx = g["indices"][:10]
    for n_axes in (1, 5, 64, 130):
        axes = np.resize(g["axes"], (n_axes, 3))
        code, out = call(lib, centers, axes, pot.images, g["offsets"], pot.coeff12, pot.coeff6,
                         pot.shift, pot.floor2, starts, idx, float(g["cutoff2"]))
        ocode, ref = call(type("L", (), {"evaluate_reused_neighbors":
                                         oracle.load().oracle_reused_neighbors})(), centers, axes,
                          pot.images, g["offsets"], pot.coeff12, pot.coeff6, pot.shift,
                          pot.floor2, starts, idx, float(g["cutoff2"]))
        assert code == ocode == 0
        np.testing.assert_array_equal(out, ref)
        assert (out[0] == 0).all() and (out[2] == 0).all()
