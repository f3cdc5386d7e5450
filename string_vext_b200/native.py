"""``NativeReusePotential``: the reference's CPU driver interface, with the
pair sum in this project's CUDA library.

Mirrors src/string_vext/native.py:12-68 (and the ReusePotential /
TriclinicSitePotential set-up it inherits, neighbor.py:9-30,
physics.py:43-57): the same constructor arguments, the same image set and
per-image coefficients, 512-center batches with a cKDTree ball query at
cutoff + max|offset|, a CSR list and one ``evaluate_reused_neighbors`` call
per batch, the same ``RuntimeError`` on a nonzero status and ``ValueError`` on
non-finite output, and the same ``query_seconds``/``compute_seconds``
counters.  The only change is the default library: ``libvext_b200.so``,
whose ``evaluate_reused_neighbors`` evaluates the batch on the GPU and returns
bit-identical FP64 energies.  Passing ``library=`` any other build of the
reference kernel keeps working.
"""
from __future__ import annotations

import ctypes
import itertools
import time
from pathlib import Path

import numpy as np

from . import _lib
from .physics import body_offsets, require_identical_sites, validate_case


class NativeReusePotential:
    def __init__(self, case: dict, library: Path | str | None = None, batch_size: int = 512):
        from scipy.spatial import cKDTree
        validate_case(case)
        require_identical_sites(case)
        if batch_size < 1:
            raise ValueError("positive center batch required")
        self.case = case
        self.offsets = np.ascontiguousarray(body_offsets(case))
        self.cutoff = float(case["cutoff"])
        self.radius = self.cutoff + float(np.abs(self.offsets).max())
        cell = np.asarray(case["cell"], dtype=np.float64)
        self.cell = cell
        inverse = np.linalg.inv(cell)
        spacing = 1 / np.linalg.norm(inverse, axis=0)
        reach = np.ceil(self.radius / spacing).astype(int) + 1
        shifts = np.array(list(itertools.product(*[range(-r, r + 1) for r in reach])), dtype=float)
        atoms = np.mod(case["frame_frac"], 1)
        self.images = np.ascontiguousarray((atoms[None] + shifts[:, None]).reshape(-1, 3) @ cell)
        sigma = np.tile(case["frame_sigma"], len(shifts))
        epsilon = np.tile(case["frame_epsilon"], len(shifts))
        mixed_sigma = (sigma + case["guest_sigma"][0]) / 2
        mixed_epsilon = np.sqrt(epsilon * case["guest_epsilon"][0])
        sigma6 = mixed_sigma**6
        self.coeff12 = np.ascontiguousarray(4 * mixed_epsilon * sigma6**2)
        self.coeff6 = np.ascontiguousarray(4 * mixed_epsilon * sigma6)
        cut6 = (mixed_sigma / self.cutoff)**6
        self.shift = np.ascontiguousarray(-4 * mixed_epsilon * (cut6**2 - cut6))
        self.floor2 = np.ascontiguousarray((.1 * mixed_sigma)**2)
        self.tree = cKDTree(self.images)
        self.batch_size = batch_size
        if library is None:
            self.library = _lib.load()
        else:
            self.library = ctypes.CDLL(str(Path(library).resolve()))
        self.kernel = self.library.evaluate_reused_neighbors
        self.kernel.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_double] + [ctypes.c_void_p] * 11
        self.kernel.restype = ctypes.c_int
        self.query_seconds = 0.
        self.compute_seconds = 0.
        self.neighbor_queries = 0
        self.max_neighbors = 0

    def evaluate(self, centers: np.ndarray, axes: np.ndarray) -> np.ndarray:
        centers, axes = np.asarray(centers, dtype=float), np.asarray(axes, dtype=float)
        if (centers.ndim != 2 or centers.shape[1] != 3
                or axes.ndim != 2 or axes.shape[1] != 3
                or not np.isfinite(centers).all() or not np.isfinite(axes).all()
                or (np.linalg.norm(axes, axis=1) <= 0).any()):
            raise ValueError("finite fractional centers and nonzero directors required")
        axes = np.ascontiguousarray(axes / np.linalg.norm(axes, axis=1, keepdims=True))
        cart = np.ascontiguousarray(np.mod(centers, 1) @ self.cell)
        output = np.empty((len(centers), len(axes)), dtype=np.float64)
        buffers = (self.images, self.offsets, self.coeff12, self.coeff6, self.shift, self.floor2)
        for start in range(0, len(cart), self.batch_size):
            end = min(start + self.batch_size, len(cart))
            stamp = time.perf_counter()
            groups = self.tree.query_ball_point(cart[start:end], self.radius, workers=1)
            lengths = np.fromiter((len(g) for g in groups), dtype=np.int64, count=len(groups))
            starts = np.empty(len(groups) + 1, dtype=np.int64)
            starts[0] = 0
            starts[1:] = np.cumsum(lengths)
            indices = (np.concatenate([np.asarray(g, dtype=np.int32) for g in groups])
                       if starts[-1] else np.empty(0, np.int32))
            self.neighbor_queries += len(groups)
            self.max_neighbors = max(self.max_neighbors, int(lengths.max(initial=0)))
            self.query_seconds += time.perf_counter() - stamp
            stamp = time.perf_counter()
            arrays = (cart[start:end], axes, *buffers, starts, indices, output[start:end])
            result = self.kernel(len(groups), len(axes), len(self.images), self.cutoff**2,
                                 *(a.ctypes.data_as(ctypes.c_void_p) for a in arrays))
            if result:
                raise RuntimeError(f"native neighbor kernel failed with code {result}")
            self.compute_seconds += time.perf_counter() - stamp
        if not np.isfinite(output).all():
            raise ValueError("nonfinite native Vext energy")
        return output
