"""evaluate_reused_neighbors_noalloc through the C ABI.

That entry point serves callers that may not allocate GPU memory (plug-ins
whose host runtime owns the GPU memory budget, real-time loops that cannot
take an allocation's synchronisation): it keeps its scratch in a fixed
64 MiB device array inside the library instead of cudaMalloc'd buffers.  Its
results must be the regular drop-in's results -- here bit for bit, the
tolerance every drop-in test uses -- on two calls in a row (the second call
finds the first call's leftovers in the shared array), repeated calls must
not change the device's free memory, and an over-sized batch must be refused
before anything is copied to the device.  This file is collected last so
that a failure here never hides another test's result.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from string_vext_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _call(fn, centers, axes, pot, offsets, starts, indices, cutoff2, n_images=None):
    out = np.full((len(centers), len(axes)), -7.0)
    arrays = [np.ascontiguousarray(a) for a in (centers, axes, pot.images, offsets, pot.coeff12,
                                                 pot.coeff6, pot.shift, pot.floor2)]
    s = np.ascontiguousarray(starts, dtype=np.int64)
    i = np.ascontiguousarray(indices, dtype=np.int32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    code = fn(len(centers), len(axes), len(pot.images) if n_images is None else n_images,
              cutoff2, *(p(a) for a in arrays), p(s), p(i), p(out))
    return code, out


def test_noalloc_matches_regular_entry_on_two_calls(golden):
    g = golden("csr_batch.npz")
    lib = _lib.load()
    pot = oracle.ReferenceDriver(synth.small_field(), _lib.LIB_PATH)
    args = (g["centers"], g["axes"], pot, g["offsets"], g["starts"], g["indices"],
            float(g["cutoff2"]))
    code, regular = _call(lib.evaluate_reused_neighbors, *args)
    assert code == 0
    np.testing.assert_array_equal(regular, g["output"])
    for _ in range(2):
        code, static = _call(lib.evaluate_reused_neighbors_noalloc, *args)
        assert code == 0
        np.testing.assert_array_equal(static, regular)
    # a smaller second batch after a larger one: leftovers must not leak in
    half = len(g["centers"]) // 2
    small = (g["centers"][:half], g["axes"][:5], pot, g["offsets"], g["starts"][:half + 1],
             g["indices"], float(g["cutoff2"]))
    code_r, reg_small = _call(lib.evaluate_reused_neighbors, *small)
    code_s, st_small = _call(lib.evaluate_reused_neighbors_noalloc, *small)
    assert code_r == code_s == 0
    np.testing.assert_array_equal(st_small, reg_small)


def test_noalloc_leaves_device_free_memory_unchanged(golden):
    """After one call has loaded the module, further calls allocate nothing:
    the device's free memory (cudaMemGetInfo) is the same before and after."""
    torch = pytest.importorskip("torch")
    g = golden("csr_batch.npz")
    lib = _lib.load()
    pot = oracle.ReferenceDriver(synth.small_field(), _lib.LIB_PATH)
    args = (g["centers"], g["axes"], pot, g["offsets"], g["starts"], g["indices"],
            float(g["cutoff2"]))
    code, first = _call(lib.evaluate_reused_neighbors_noalloc, *args)
    assert code == 0
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        code, again = _call(lib.evaluate_reused_neighbors_noalloc, *args)
        assert code == 0
        np.testing.assert_array_equal(again, first)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_noalloc_refuses_oversized_batches(golden):
    g = golden("csr_batch.npz")
    lib = _lib.load()
    pot = oracle.ReferenceDriver(synth.small_field(), _lib.LIB_PATH)
    # 10^6 images need ~120 MB of scratch: refused before anything is copied
    code, out = _call(lib.evaluate_reused_neighbors_noalloc, g["centers"][:1], g["axes"], pot,
                      g["offsets"], g["starts"][:2], g["indices"], float(g["cutoff2"]),
                      n_images=1_000_000)
    assert code == 19
    assert b"scratch" in lib.vext_last_error()
    assert (out == -7.0).all()
