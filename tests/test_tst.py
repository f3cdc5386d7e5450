"""Transition-state-theory post-processing of String paths (host code in the
library, no GPU): the log-domain path score against the reference's own
legacy_policy.h compiled from source (oracle/_ref/tst.so), the hopping
diffusivity against the restatement of RC_main.cu:2485-2527, and their
agreement with each other."""
import ctypes
import math

import numpy as np
import pytest

from conftest import ROOT
from oracle import string_oracle
from string_vext_b200 import _lib, synth
from string_vext_b200.tst import choose_initial, diffusivity, hop_length, log_score

REF_TST = ROOT / "oracle" / "_ref" / "tst.so"


def ref_lib():
    if not REF_TST.exists():
        pytest.skip("reference legacy_policy.h shim not built (make -C oracle ref)")
    lib = ctypes.CDLL(str(REF_TST))
    vp, cd = ctypes.c_void_p, ctypes.c_double
    lib.ref_legacy_log_score.argtypes = [vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, cd, cd, cd,
                                         ctypes.POINTER(cd)]
    lib.ref_legacy_log_score.restype = ctypes.c_int
    lib.ref_legacy_choose_initial.argtypes = [ctypes.c_int, cd, ctypes.c_int, cd]
    lib.ref_legacy_choose_initial.restype = ctypes.c_int
    return lib


def ref_score(lib, path, energy, cell, T, mass, hop):
    p = np.asarray(path, dtype=float)
    cols = [np.ascontiguousarray(p[:, k]) for k in range(3)]
    rows = [np.ascontiguousarray(np.asarray(cell, dtype=float)[:, k]) for k in range(3)]
    e = np.ascontiguousarray(energy, dtype=float)
    out = ctypes.c_double()
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    valid = lib.ref_legacy_log_score(*(ptr(c) for c in cols), ptr(e), len(e),
                                     *(ptr(r) for r in rows), T, mass, hop, ctypes.byref(out))
    return bool(valid), out.value


def paths(n_paths=12, seed=11):
    rng = np.random.default_rng(seed)
    case = synth.small_field()
    for _ in range(n_paths):
        n = int(rng.integers(8, 96))
        t = np.linspace(0, 1, n)[:, None]
        start = rng.random(3)
        frac = start + t * (np.array([0.0, 0.0, 1.0]) + 0.05 * rng.normal(size=3))
        frac += 0.01 * rng.normal(size=frac.shape)
        energy = rng.uniform(-3000.0, 4000.0, n)
        yield case, frac, energy


def test_log_score_matches_reference_header():
    lib = ref_lib()
    for case, frac, energy in paths():
        for T, mass, hop in ((298.0, 30.07, 15.0), (77.0, 28.05, hop_length(case, 3))):
            ours = log_score(frac, energy, case["cell"], T, mass, hop)
            ref = ref_score(lib, frac, energy, case["cell"], T, mass, hop)
            assert ours[0] == ref[0]
            assert ours[1] == pytest.approx(ref[1], rel=1e-14, abs=1e-12)


def test_log_score_invalid_inputs_match_reference():
    lib = ref_lib()
    case, frac, energy = next(paths(1))
    bad_energy = energy.copy()
    bad_energy[3] = np.nan
    for args in ((frac[:1], energy[:1], 298.0, 30.0, 10.0),
                 (frac, energy, 0.0, 30.0, 10.0),
                 (frac, energy, 298.0, -1.0, 10.0),
                 (frac, energy, 298.0, 30.0, 0.0),
                 (frac, bad_energy, 298.0, 30.0, 10.0)):
        f, e, T, m, h = args
        assert log_score(f, e, case["cell"], T, m, h)[0] is False
        assert ref_score(lib, f, e, case["cell"], T, m, h)[0] is False


def test_choose_initial_matches_reference():
    lib = ref_lib()
    for vi in (False, True):
        for vf in (False, True):
            for li, lf in ((-20.0, -25.0), (-25.0, -20.0), (-20.0, -20.0)):
                assert choose_initial((vi, li), (vf, lf)) == bool(
                    lib.ref_legacy_choose_initial(int(vi), li, int(vf), lf))


def test_diffusivity_matches_restatement_and_log_score():
    for case, frac, energy in paths():
        hop = hop_length(case, 3)
        d0 = diffusivity(frac, energy, case["cell"], hop, 298.0, 30.07)
        ref = string_oracle.tst_diffusivity(frac, energy, case["cell"], hop, 298.0, 30.07)
        assert d0 == pytest.approx(ref, rel=1e-13)
        valid, logd = log_score(frac, energy, case["cell"], 298.0, 30.07, hop)
        assert valid
        # the same TST formula in the log domain (energies far below the 600 T cap)
        assert math.log(d0) == pytest.approx(logd, rel=1e-10, abs=1e-9)


def test_diffusivity_rejects_bad_arguments():
    case, frac, energy = next(paths(1))
    with pytest.raises(_lib.VextError):
        diffusivity(frac[:1], energy[:1], case["cell"], 10.0, 298.0, 30.0)
    with pytest.raises(_lib.VextError):
        diffusivity(frac, energy, case["cell"], 10.0, -1.0, 30.0)
