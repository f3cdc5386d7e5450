"""``VextSystem``: one framework + one symmetric two-site guest on the GPU.

A thin owner of a ``vext_system`` handle (include/vext_b200.h).  All compute
goes through the CUDA library; this class only marshals arrays.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .physics import body_offsets, require_identical_sites, validate_case


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


class VextSystem:
    """Device-resident framework + guest.  ``case`` uses the reference's case
    dictionary layout (src/string_vext/input.py:49-55)."""

    def __init__(self, case: dict):
        validate_case(case)
        require_identical_sites(case)
        self.case = case
        self.cell = _c(case["cell"])
        self.offsets = _c(body_offsets(case))
        self._frac = _c(case["frame_frac"])
        self._sigma = _c(case["frame_sigma"])
        self._eps = _c(case["frame_epsilon"])
        desc = _lib.SystemDesc()
        desc.cell[:] = self.cell.reshape(-1).tolist()
        desc.n_atoms = len(self._frac)
        desc.frac = self._frac.ctypes.data
        desc.sigma = self._sigma.ctypes.data
        desc.epsilon = self._eps.ctypes.data
        desc.guest_sigma = float(case["guest_sigma"][0])
        desc.guest_epsilon = float(case["guest_epsilon"][0])
        desc.offsets[:] = self.offsets.tolist()
        desc.cutoff = float(case["cutoff"])
        desc.temperature = float(case["temperature"])
        handle = ctypes.c_void_p()
        self._lib = _lib.load()
        _lib.check(self._lib.vext_system_create(ctypes.byref(desc), ctypes.byref(handle)))
        self.handle = handle
        self.last_stats: dict | None = None

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.vext_system_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def invalidate(self) -> None:
        """Drop cached region lists (the next call rebuilds them)."""
        _lib.check(self._lib.vext_system_invalidate(self.handle))

    def last_timings(self) -> dict:
        """Device ms of the last list build, near and far pair kernels, epilogue."""
        vals = [ctypes.c_double() for _ in range(4)]
        _lib.check(self._lib.vext_last_timings(self.handle, *(ctypes.byref(v) for v in vals)))
        return {"list_ms": vals[0].value, "near_ms": vals[1].value, "far_ms": vals[2].value,
                "epilogue_ms": vals[3].value}

    def count_pairs(self, size: int, axes, r_split: float = 0.0) -> tuple[int, int]:
        """Exact in-cutoff (site, image) pairs of the size^3 x len(axes) field:
        (all pairs, pairs the FP32 far kernel evaluates at this r_split)."""
        axes = _c(axes)
        total, far = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(self._lib.vext_count_pairs(self.handle, size, len(axes), _lib.ptr(axes),
                                              float(r_split), ctypes.byref(total),
                                              ctypes.byref(far)))
        return total.value, far.value

    # ------------------------------------------------------------------ field
    def field(self, size: int, axes, mode: int = _lib.VEXT_MODE_MIXED,
              orientation: bool = True, energy: bool = False, marginal: bool = False,
              site: bool = False, grid: bool = False, **opts) -> dict:
        """Vext field on the size^3 grid x unit directors ``axes`` (host arrays).
        Returns the requested channels in the reference layout."""
        axes = _c(axes)
        n_axes = len(axes)
        s3 = size ** 3
        out = {}
        o_k = np.empty((n_axes, size, size, size), np.float32) if orientation else None
        e64 = np.empty((s3, n_axes), np.float64) if energy else None
        m_k = np.empty((size, size, size), np.float32) if marginal else None
        s_k = np.empty((2, size, size, size), np.float32) if site else None
        g_k = np.empty((size, size, size), np.float32) if grid else None
        stats = _lib.FieldStats()
        opt = _lib.options(mode, **opts)
        _lib.check(self._lib.vext_field(self.handle, size, n_axes, _lib.ptr(axes),
                                        ctypes.byref(opt), _lib.ptr(o_k), _lib.ptr(e64),
                                        _lib.ptr(m_k), _lib.ptr(s_k), _lib.ptr(g_k),
                                        ctypes.byref(stats)))
        self.last_stats = stats.as_dict()
        for key, value in (("orientation_K", o_k), ("energy", e64), ("marginal_K", m_k),
                           ("site_K", s_k), ("grid", g_k)):
            if value is not None:
                out[key] = value
        return out

    def field_device(self, size: int, axes, out_orientation, mode: int = _lib.VEXT_MODE_MIXED,
                     out_energy=None, out_marginal=None, out_site=None, out_grid=None,
                     stream=None, **opts) -> None:
        """Device-pointer variant: outputs are CUDA tensors (float32 [O, S, S, S]
        etc.), work is enqueued on ``stream`` (a torch.cuda.Stream or None)."""
        axes = _c(axes)
        opt = _lib.options(mode, **opts)
        handle = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _lib.check(self._lib.vext_field_device(self.handle, size, len(axes), _lib.ptr(axes),
                                               ctypes.byref(opt), _lib.ptr(out_orientation),
                                               _lib.ptr(out_energy), _lib.ptr(out_marginal),
                                               _lib.ptr(out_site), _lib.ptr(out_grid), handle))

    def field_adjoint(self, size: int, axes, mode: int = _lib.VEXT_MODE_MIXED,
                      pinned: bool = False, **opts):
        """Forward + adjoint over the field poses (host arrays).  Returns the
        float32 energy [O, S, S, S] and gradient [O, S, S, S, 6] = (dE/dcenter,
        dE/du projected on the plane normal to u).  ``pinned=True`` returns
        them in page-locked memory (torch's pinned host allocator), which the
        kernels of the mixed mode write directly: the call then costs about
        the device time instead of device time plus a copy."""
        axes = _c(axes)
        n_axes = len(axes)
        if pinned:
            import torch
            energy = torch.empty((n_axes, size, size, size), dtype=torch.float32,
                                 pin_memory=True).numpy()
            grad = torch.empty((n_axes, size, size, size, 6), dtype=torch.float32,
                               pin_memory=True).numpy()
        else:
            energy = np.empty((n_axes, size, size, size), np.float32)
            grad = np.empty((n_axes, size, size, size, 6), np.float32)
        opt = _lib.options(mode, **opts)
        _lib.check(self._lib.vext_field_adjoint(self.handle, size, n_axes, _lib.ptr(axes),
                                                ctypes.byref(opt), _lib.ptr(energy),
                                                _lib.ptr(grad)))
        return energy, grad

    def field_adjoint_device(self, size: int, axes, energy=None, gradient=None,
                             energy_f64=None, gradient_f64=None,
                             mode: int = _lib.VEXT_MODE_MIXED, stream=None, **opts) -> None:
        """Device-pointer variant (CUDA tensors, [O, S, S, S] and [O, S, S, S, 6]);
        the mixed mode writes float32 outputs, the FP64 modes any of the four."""
        axes = _c(axes)
        opt = _lib.options(mode, **opts)
        handle = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _lib.check(self._lib.vext_field_adjoint_device(
            self.handle, size, len(axes), _lib.ptr(axes), ctypes.byref(opt), _lib.ptr(energy),
            _lib.ptr(gradient), _lib.ptr(energy_f64), _lib.ptr(gradient_f64), handle))

    # ------------------------------------------------------------------ poses
    def pose_energy_grad(self, centers, quats, mode: int = _lib.VEXT_MODE_MIXED,
                         grad: bool = True, **opts):
        """Host arrays: centers (n, 3) Cartesian A, quats (n, 4) (w, x, y, z).
        Returns energy (n,), dE/dcenter (n, 3), dE/dq (n, 4), dE/du (n, 3)."""
        centers, quats = _c(centers), _c(quats)
        n = len(centers)
        e = np.empty(n)
        gc = np.empty((n, 3)) if grad else None
        gq = np.empty((n, 4)) if grad else None
        gu = np.empty((n, 3)) if grad else None
        opt = _lib.options(mode, **opts)
        _lib.check(self._lib.vext_pose_energy_grad(self.handle, n, _lib.ptr(centers),
                                                   _lib.ptr(quats), ctypes.byref(opt),
                                                   _lib.ptr(e), _lib.ptr(gc), _lib.ptr(gq),
                                                   _lib.ptr(gu)))
        return e, gc, gq, gu

    def pose_energy_grad_device(self, centers, quats, energy, grad_center=None, grad_quat=None,
                                grad_director=None, mode: int = _lib.VEXT_MODE_MIXED,
                                stream=None, **opts) -> None:
        """CUDA float64 tensors in and out, enqueued on ``stream``."""
        opt = _lib.options(mode, **opts)
        handle = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _lib.check(self._lib.vext_pose_energy_grad_device(
            self.handle, int(centers.shape[0]), _lib.ptr(centers), _lib.ptr(quats),
            ctypes.byref(opt), _lib.ptr(energy), _lib.ptr(grad_center), _lib.ptr(grad_quat),
            _lib.ptr(grad_director), handle))


class VextBatch:
    """Many systems' fields in one persistent, graph-captured launch
    (``vext_batch_create``).  ``outputs`` are CUDA float32 tensors
    [n_axes, S, S, S], one per system; ``run()`` replays the graph."""

    def __init__(self, systems, size: int, axes, outputs, gradients=None, **opts):
        self._lib = _lib.load()
        self.systems = list(systems)           # kept alive: the batch points into them
        self.outputs = list(outputs)
        self.gradients = list(gradients) if gradients is not None else None
        self.axes = _c(axes)
        handles = (ctypes.c_void_p * len(self.systems))(*[s.handle.value for s in self.systems])
        outs = (ctypes.c_void_p * len(self.outputs))(*[o.data_ptr() for o in self.outputs])
        opt = _lib.options(_lib.VEXT_MODE_MIXED, **opts)
        handle = ctypes.c_void_p()
        if self.gradients is None:
            _lib.check(self._lib.vext_batch_create(len(self.systems), handles, size,
                                                   len(self.axes), _lib.ptr(self.axes),
                                                   ctypes.byref(opt), outs,
                                                   ctypes.byref(handle)))
        else:
            grads = (ctypes.c_void_p * len(self.gradients))(
                *[g.data_ptr() for g in self.gradients])
            _lib.check(self._lib.vext_batch_create_adjoint(len(self.systems), handles, size,
                                                           len(self.axes), _lib.ptr(self.axes),
                                                           ctypes.byref(opt), outs, grads,
                                                           ctypes.byref(handle)))
        self.handle = handle

    def run(self, stream=None) -> None:
        h = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _lib.check(self._lib.vext_batch_run(self.handle, h))

    def check(self) -> None:
        _lib.check(self._lib.vext_batch_status(self.handle))

    def info(self) -> dict:
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        d, e = ctypes.c_int(), ctypes.c_int()
        _lib.check(self._lib.vext_batch_info(self.handle, ctypes.byref(a), ctypes.byref(b),
                                             ctypes.byref(c), ctypes.byref(d), ctypes.byref(e)))
        tuning = self.tuning()
        name = next((t["name"] for t in tuning
                     if t["shape"] == d.value and t["grid"] == e.value), None)
        return {"work_items": a.value, "poses": b.value, "list_bytes": c.value,
                "shape": d.value, "cta_shape": name, "grid": e.value,
                "adjoint": self.gradients is not None, "tuning": tuning}

    def refined(self) -> int:
        """Poses the last replay re-evaluated in FP64 (waits for the device)."""
        n = ctypes.c_int64()
        _lib.check(self._lib.vext_batch_refined(self.handle, ctypes.byref(n)))
        return n.value

    def tuning(self) -> list:
        """The autotuner's candidates: shape name (threads x directors per
        thread[/CTAs-per-SM bound]), resident CTAs, sample time (ms)."""
        m = 16
        n = ctypes.c_int()
        shapes, grids = (ctypes.c_int * m)(), (ctypes.c_int * m)()
        ms, names = (ctypes.c_float * m)(), (ctypes.c_char_p * m)()
        _lib.check(self._lib.vext_batch_tuning(self.handle, m, ctypes.byref(n), shapes, grids,
                                               ms, names))
        return [{"name": names[i].decode(), "shape": shapes[i], "grid": grids[i],
                 "sample_ms": ms[i]} for i in range(min(n.value, m))]

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.vext_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VextPoseBatch:
    """Poses of many systems (e.g. one String path per framework x guest)
    forward + adjoint in one launch (``vext_pose_batch_create``).  ``counts[k]``
    poses belong to ``systems[k]``; ``run`` takes CUDA float64 tensors with the
    poses of all systems stacked in that order."""

    def __init__(self, systems, counts, mode: int = _lib.VEXT_MODE_MIXED, **opts):
        self._lib = _lib.load()
        self.systems = list(systems)           # kept alive: the batch points into them
        offsets = np.zeros(len(self.systems) + 1, dtype=np.int64)
        offsets[1:] = np.cumsum(np.asarray(counts, dtype=np.int64))
        self.n = int(offsets[-1])
        handles = (ctypes.c_void_p * len(self.systems))(*[s.handle.value for s in self.systems])
        opt = _lib.options(mode, **opts)
        handle = ctypes.c_void_p()
        _lib.check(self._lib.vext_pose_batch_create(len(self.systems), handles,
                                                    _lib.ptr(offsets), ctypes.byref(opt),
                                                    ctypes.byref(handle)))
        self.handle = handle

    def run(self, centers, quats, energy, grad_center=None, grad_quat=None,
            grad_director=None, stream=None) -> None:
        h = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _lib.check(self._lib.vext_pose_batch_run(self.handle, _lib.ptr(centers), _lib.ptr(quats),
                                                 _lib.ptr(energy), _lib.ptr(grad_center),
                                                 _lib.ptr(grad_quat), _lib.ptr(grad_director),
                                                 h))

    def check(self) -> None:
        _lib.check(self._lib.vext_pose_batch_status(self.handle))

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.vext_pose_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
