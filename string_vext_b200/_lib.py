"""ctypes binding of ``libvext_b200.so`` (the sm_100a library, C ABI in
include/vext_b200.h).

The library is built in-tree (``string_vext_b200/lib``); there is no CPU
fallback: importing the bindings without the library, or calling a compute
entry without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PACKAGE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("VEXT_B200_LIBRARY", PACKAGE / "lib" / "libvext_b200.so"))

VEXT_MODE_MIXED = 0
VEXT_MODE_FP64 = 1
VEXT_MODE_FP64_PLAIN = 2
VEXT_MODE_FP32_NAIVE = 3

VEXT_ERR_TIMEOUT = 17
VEXT_ERR_ARGUMENT = 18
VEXT_ERR_CAPACITY = 19

STATUS = {0: "ok", 1: "bad sizes", 2: "CSR starts decreasing", 3: "CSR index out of range",
          4: "non-finite energy", 16: "CUDA error", 17: "device wait timeout",
          18: "invalid argument", 19: "capacity exceeded", 20: "out of memory"}


class SystemDesc(ctypes.Structure):
    _fields_ = [("cell", ctypes.c_double * 9), ("n_atoms", ctypes.c_int),
                ("frac", ctypes.c_void_p), ("sigma", ctypes.c_void_p),
                ("epsilon", ctypes.c_void_p), ("guest_sigma", ctypes.c_double),
                ("guest_epsilon", ctypes.c_double), ("offsets", ctypes.c_double * 2),
                ("cutoff", ctypes.c_double), ("temperature", ctypes.c_double)]


class Options(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("r_split", ctypes.c_double),
                ("band_lo", ctypes.c_double), ("band_hi", ctypes.c_double),
                ("centers_per_region", ctypes.c_int), ("variant", ctypes.c_int),
                ("batch_shape", ctypes.c_int), ("reserved", ctypes.c_int * 2)]


class FieldStats(ctypes.Structure):
    _fields_ = [("poses", ctypes.c_int64), ("regions", ctypes.c_int64),
                ("list_entries", ctypes.c_int64), ("near_entries", ctypes.c_int64),
                ("refined_poses", ctypes.c_int64), ("list_build_ms", ctypes.c_double),
                ("kernel_ms", ctypes.c_double), ("epilogue_ms", ctypes.c_double),
                ("outer_entries", ctypes.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class StringParams(ctypes.Structure):
    _fields_ = [("direction", ctypes.c_int), ("delta_frac", ctypes.c_double),
                ("delta_angle_rad", ctypes.c_double), ("smooth", ctypes.c_double),
                ("rounding", ctypes.c_double), ("conv_trans_percent", ctypes.c_double),
                ("conv_rot_percent", ctypes.c_double), ("max_iterations", ctypes.c_int),
                ("check_every", ctypes.c_int), ("gradient", ctypes.c_int)]


VEXT_STRING_ANALYTIC = 0
VEXT_STRING_REFERENCE_FD = 1


class StringResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("converged_translation", ctypes.c_int), ("converged_rotation", ctypes.c_int),
                ("movement_translation", ctypes.c_double),
                ("movement_rotation", ctypes.c_double),
                ("threshold_translation", ctypes.c_double),
                ("threshold_rotation", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class VextError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"vext_b200 status {code} ({STATUS.get(code, '?')}): {message}")
        self.code = code


_lib = None


def load(path=None) -> ctypes.CDLL:
    """Load the library once; raise if it is missing (no fallback).  ``path``
    selects another build of the library; it must be given before the first
    load of the process."""
    global _lib, LIB_PATH
    if path is not None and Path(path).resolve() != LIB_PATH.resolve():
        if _lib is not None:
            raise RuntimeError(f"vext_b200 library already loaded from {LIB_PATH}")
        LIB_PATH = Path(path)
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"vext_b200 CUDA library not built: {LIB_PATH} "
                           "(run __graft_entry__.build() or make -C string_vext_b200/csrc)")
    lib = ctypes.CDLL(str(LIB_PATH))
    vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.evaluate_reused_neighbors.argtypes = [ci, ci, ci, cd] + [vp] * 11
    lib.evaluate_reused_neighbors.restype = ci
    lib.evaluate_reused_neighbors_noalloc.argtypes = [ci, ci, ci, cd] + [vp] * 11
    lib.evaluate_reused_neighbors_noalloc.restype = ci
    lib.vext_last_error.argtypes = []
    lib.vext_last_error.restype = ctypes.c_char_p
    lib.vext_check_wait_timeout.argtypes = [ci]
    lib.vext_check_wait_timeout.restype = ci
    lib.vext_version.argtypes = []
    lib.vext_version.restype = ctypes.c_char_p
    lib.vext_default_options.argtypes = [ctypes.POINTER(Options)]
    lib.vext_default_options.restype = None
    lib.vext_system_create.argtypes = [ctypes.POINTER(SystemDesc), ctypes.POINTER(vp)]
    lib.vext_system_create.restype = ci
    lib.vext_system_destroy.argtypes = [vp]
    lib.vext_system_destroy.restype = ci
    lib.vext_field.argtypes = [vp, ci, ci, vp, ctypes.POINTER(Options), vp, vp, vp, vp, vp,
                               ctypes.POINTER(FieldStats)]
    lib.vext_field.restype = ci
    lib.vext_field_device.argtypes = [vp, ci, ci, vp, ctypes.POINTER(Options), vp, vp, vp, vp,
                                      vp, vp]
    lib.vext_field_device.restype = ci
    lib.vext_pose_energy_grad.argtypes = [vp, ci, vp, vp, ctypes.POINTER(Options), vp, vp, vp, vp]
    lib.vext_pose_energy_grad.restype = ci
    lib.vext_pose_energy_grad_device.argtypes = [vp, ci, vp, vp, ctypes.POINTER(Options), vp, vp,
                                                 vp, vp, vp]
    lib.vext_pose_energy_grad_device.restype = ci
    lib.vext_system_invalidate.argtypes = [vp]
    lib.vext_system_invalidate.restype = ci
    lib.vext_last_timings.argtypes = [vp] + [ctypes.POINTER(ctypes.c_double)] * 4
    lib.vext_last_timings.restype = ci
    lib.vext_count_pairs.argtypes = [vp, ci, ci, vp, cd, ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(ctypes.c_int64)]
    lib.vext_count_pairs.restype = ci
    lib.vext_batch_create.argtypes = [ci, vp, ci, ci, vp, ctypes.POINTER(Options), vp,
                                      ctypes.POINTER(vp)]
    lib.vext_batch_create.restype = ci
    lib.vext_batch_create_adjoint.argtypes = [ci, vp, ci, ci, vp, ctypes.POINTER(Options), vp,
                                              vp, ctypes.POINTER(vp)]
    lib.vext_batch_create_adjoint.restype = ci
    lib.vext_field_adjoint_device.argtypes = [vp, ci, ci, vp, ctypes.POINTER(Options), vp, vp,
                                              vp, vp, vp]
    lib.vext_field_adjoint_device.restype = ci
    lib.vext_field_adjoint.argtypes = [vp, ci, ci, vp, ctypes.POINTER(Options), vp, vp]
    lib.vext_field_adjoint.restype = ci
    lib.vext_batch_tuning.argtypes = [vp, ci, ctypes.POINTER(ci), ctypes.POINTER(ci),
                                      ctypes.POINTER(ci), ctypes.POINTER(ctypes.c_float),
                                      ctypes.POINTER(ctypes.c_char_p)]
    lib.vext_batch_tuning.restype = ci
    lib.vext_pose_batch_create.argtypes = [ci, vp, vp, ctypes.POINTER(Options),
                                           ctypes.POINTER(vp)]
    lib.vext_pose_batch_create.restype = ci
    lib.vext_pose_batch_run.argtypes = [vp] + [vp] * 6 + [vp]
    lib.vext_pose_batch_run.restype = ci
    lib.vext_pose_batch_status.argtypes = [vp]
    lib.vext_pose_batch_status.restype = ci
    lib.vext_pose_batch_destroy.argtypes = [vp]
    lib.vext_pose_batch_destroy.restype = ci
    lib.vext_tst_diffusivity.argtypes = [ci, vp, vp, vp, cd, cd, cd,
                                         ctypes.POINTER(ctypes.c_double)]
    lib.vext_tst_diffusivity.restype = ci
    lib.vext_tst_log_score.argtypes = [ci, vp, vp, vp, cd, cd, cd, ctypes.POINTER(ci),
                                       ctypes.POINTER(ctypes.c_double)]
    lib.vext_tst_log_score.restype = ci
    lib.vext_batch_run.argtypes = [vp, vp]
    lib.vext_batch_run.restype = ci
    lib.vext_batch_status.argtypes = [vp]
    lib.vext_batch_status.restype = ci
    lib.vext_batch_destroy.argtypes = [vp]
    lib.vext_batch_destroy.restype = ci
    lib.vext_batch_info.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int64)] * 3 + \
        [ctypes.POINTER(ci)] * 2
    lib.vext_batch_info.restype = ci
    lib.vext_batch_refined.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    lib.vext_batch_refined.restype = ci
    lib.vext_string_default_params.argtypes = [ctypes.POINTER(StringParams)]
    lib.vext_string_default_params.restype = None
    lib.vext_string_run.argtypes = [vp, ci, vp, vp, ctypes.POINTER(StringParams),
                                    ctypes.POINTER(Options), ctypes.POINTER(StringResult)]
    lib.vext_string_run.restype = ci
    lib.vext_measure_pipes.argtypes = [ci] + [ctypes.POINTER(ctypes.c_double)] * 3
    lib.vext_measure_pipes.restype = ci
    lib.vext_measure_fp32_peak.argtypes = [ci, ctypes.POINTER(ctypes.c_double)]
    lib.vext_measure_fp32_peak.restype = ci
    _lib = lib
    return lib


def check(code: int) -> None:
    if code:
        message = load().vext_last_error().decode(errors="replace")
        raise VextError(code, message)


def ptr(array) -> ctypes.c_void_p | None:
    """Data pointer of a numpy array or torch tensor (None passes NULL)."""
    if array is None:
        return None
    if isinstance(array, np.ndarray):
        return ctypes.c_void_p(array.ctypes.data)
    return ctypes.c_void_p(array.data_ptr())


def options(mode: int = VEXT_MODE_MIXED, r_split: float | None = None,
            band: tuple[float, float] | None = None,
            centers_per_region: int | None = None, variant: int | None = None,
            batch_shape: int | None = None) -> Options:
    opt = Options()
    load().vext_default_options(ctypes.byref(opt))
    opt.mode = mode
    if r_split is not None:
        opt.r_split = r_split
    if band is not None:
        opt.band_lo, opt.band_hi = band
    if centers_per_region is not None:
        opt.centers_per_region = centers_per_region
    if variant is not None:
        opt.variant = variant
    if batch_shape is not None:
        opt.batch_shape = batch_shape
    return opt


def version() -> str:
    return load().vext_version().decode()


def measure_fp32_peak(iterations: int = 20000) -> float:
    value = ctypes.c_double()
    check(load().vext_measure_fp32_peak(iterations, ctypes.byref(value)))
    return value.value


def measure_pipes(iterations: int = 20000) -> dict:
    """FFMA, FFMA2 (counted per FMA) and RCP throughput of the current GPU."""
    vals = [ctypes.c_double() for _ in range(3)]
    check(load().vext_measure_pipes(iterations, *(ctypes.byref(v) for v in vals)))
    return {"ffma_per_s": vals[0].value, "ffma2_fma_per_s": vals[1].value,
            "rcp_per_s": vals[2].value}
