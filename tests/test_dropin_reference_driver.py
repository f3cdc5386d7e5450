"""The drop-in through the reference's own, unmodified Python driver.

The reference package (``string_vext``: ``calculate_vext``,
``NativeReusePotential``; src/string_vext/vext.py:21-43, native.py:12-68) is
installed, unchanged, into ``baseline/_ref`` by

    python -m pip install --no-index --no-build-isolation --no-deps \
        --target baseline/_ref <copy of the reference checkout>

Its driver binds ``evaluate_reused_neighbors`` of whatever library it is
given (``kernel=``, the CLI's ``--kernel``).  Given this project's
``libvext_b200.so``, every output channel must equal, bit for bit, what the
same driver produced with the reference kernel built from source (the golden
fixtures of tests/golden/make_golden.py).  Skipped when the package is not
installed.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from string_vext_b200 import _lib, synth

pytestmark = pytest.mark.gpu

REF_PACKAGE = Path(__file__).resolve().parents[1] / "baseline" / "_ref"


@pytest.fixture(scope="module")
def reference():
    if not (REF_PACKAGE / "string_vext" / "native.py").exists():
        pytest.skip("reference package not installed in baseline/_ref")
    sys.path.insert(0, str(REF_PACKAGE))
    try:
        import string_vext.native
        import string_vext.vext
    finally:
        sys.path.remove(str(REF_PACKAGE))
    assert Path(string_vext.vext.__file__).resolve().is_relative_to(REF_PACKAGE.resolve())
    return string_vext


def test_reference_calculate_vext_with_this_library(reference, golden, tmp_path):
    """calculate_vext of the reference with kernel = this library: every
    channel identical to the reference kernel's golden output."""
    g = golden("small_field_s4.npz")
    fields = reference.vext.calculate_vext(synth.small_field(), size=4, orientations=64,
                                           kernel=_lib.LIB_PATH)
    for key in ("orientation_K", "marginal_K", "site_K", "grid"):
        np.testing.assert_array_equal(fields[key], g[key], err_msg=key)
    # the skewed toy cell of the reference's unit test (beta = 115.152 deg)
    t = golden("toy_skew.npz")
    path = tmp_path / "input.dat"
    path.write_text(str(t["toy_input"]))
    toy = reference.input.parse_string_input(path)
    fields = reference.vext.calculate_vext(toy, size=3, orientations=4, kernel=_lib.LIB_PATH)
    for key in ("orientation_K", "marginal_K", "site_K", "grid", "axes"):
        np.testing.assert_array_equal(fields[key], t[f"toy_{key}"], err_msg=key)


def test_reference_driver_bit_exact_on_full_size_workloads(reference, golden):
    """NativeReusePotential of the reference with this library on sampled
    centers of the full-size and skewed workloads (edge centers included)."""
    for name, maker in (("full_field", synth.full_field), ("skewed_field", synth.skewed_field)):
        s = golden(f"{name}_sample.npz")
        driver = reference.native.NativeReusePotential(maker(), _lib.LIB_PATH)
        np.testing.assert_array_equal(driver.evaluate(s["centers"], s["axes"]), s["native"])


def test_reference_driver_raises_on_bad_input(reference):
    """The driver's own checks still fire in front of this library, and a
    kernel status would surface as its RuntimeError."""
    driver = reference.native.NativeReusePotential(synth.small_field(), _lib.LIB_PATH)
    with pytest.raises(ValueError):
        driver.evaluate(np.array([[0.1, 0.2, np.nan]]), np.eye(3))
    out = driver.evaluate(np.array([[0.1, 0.2, 0.3], [0.9, 0.5, 0.01]]), np.eye(3))
    assert out.shape == (2, 3) and np.isfinite(out).all()
