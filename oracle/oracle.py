"""ctypes/numpy front end of the FP64 oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference legs import this module, and only as the checker or the timed CPU
baseline; the product never routes through it.

Two parts:

* wrappers of ``libvext_oracle.so`` (oracle/vext_oracle.c, the plain-C FP64
  restatement of the reference arithmetic);
* ``ReferenceDriver`` -- a restatement of the reference's CPU driver
  ``NativeReusePotential`` (src/string_vext/native.py:12-68) on top of
  ``ReusePotential`` (src/string_vext/neighbor.py:9-30) and the image set of
  ``TriclinicSitePotential`` (src/string_vext/physics.py:43-57): 512-center
  batches, a cKDTree ball query at cutoff + max|offset|, a CSR neighbour list
  and one call of an ``evaluate_reused_neighbors`` library per batch.  Handed
  ``oracle/_ref/vext_kernel.so`` (the reference kernel compiled from its own
  source) it is the reference's own CPU path; handed the product library it
  exercises the drop-in boundary exactly as the reference would.
"""
from __future__ import annotations

import ctypes
import itertools
import os
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libvext_oracle.so"
REF_KERNEL = HERE / "_ref" / "vext_kernel.so"
REF_PAIR = HERE / "_ref" / "pair.so"
#: The reference's Python package, installed unchanged (pip --target) beside the repo.
REF_PACKAGE = HERE.parent / "baseline" / "_ref"

_dp = ctypes.POINTER(ctypes.c_double)
_lib = None


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        lib = ctypes.CDLL(str(LIB_PATH))
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        lib.oracle_reused_neighbors.argtypes = [ci, ci, ci, cd] + [vp] * 11
        lib.oracle_reused_neighbors.restype = ci
        lib.oracle_site_energy.argtypes = [vp, ci, vp, vp, vp, cd, cd, cd, ci, vp, vp]
        lib.oracle_site_energy.restype = ci
        lib.oracle_pose_energy.argtypes = [vp, ci, vp, vp, vp, cd, cd, vp, cd, ci, vp, ci, vp, vp]
        lib.oracle_pose_energy.restype = ci
        lib.oracle_pair_counts.argtypes = [vp, ci, vp, vp, cd, ci, vp, ci, vp, vp]
        lib.oracle_pair_counts.restype = ci
        lib.oracle_pose_energy_grad.argtypes = [vp, ci, vp, vp, vp, cd, cd, vp, cd, ci, vp, vp,
                                                vp, vp, vp]
        lib.oracle_pose_energy_grad.restype = ci
        lib.oracle_pair_lj.argtypes = [cd] * 6 + [vp] * 3 + [cd] * 5
        lib.oracle_pair_lj.restype = cd
        lib.oracle_euler_pose_energy.argtypes = [vp, ci, vp, vp, vp, ci, vp, vp, vp, cd, ci, vp, vp]
        lib.oracle_euler_pose_energy.restype = ci
        _lib = lib
    return _lib


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def body_offsets(case) -> np.ndarray:
    """Signed site offsets along the director (physics.py:88-90)."""
    xyz = np.asarray(case["guest_xyz"], dtype=float)
    mass = np.asarray(case["guest_mass"], dtype=float)
    com = (xyz * mass[:, None]).sum(0) / case["total_mass"]
    return xyz[:, 0] - com[0]


def _frame(case):
    return (_c(case["cell"]), len(case["frame_frac"]), _c(case["frame_frac"]),
            _c(case["frame_sigma"]), _c(case["frame_epsilon"]))


def pose_energy(case, centers_frac, axes) -> np.ndarray:
    """direct_pose_energy (physics.py:93-106) in FP64; axes must be unit length."""
    cell, n, frac, sig, eps = _frame(case)
    centers = _c(centers_frac)
    axes = _c(axes)
    out = np.empty((len(centers), len(axes)))
    rc = load().oracle_pose_energy(_ptr(cell), n, _ptr(frac), _ptr(sig), _ptr(eps),
                                   float(case["guest_sigma"][0]), float(case["guest_epsilon"][0]),
                                   _ptr(_c(body_offsets(case))), float(case["cutoff"]),
                                   len(centers), _ptr(centers), len(axes), _ptr(axes), _ptr(out))
    if rc:
        raise RuntimeError(f"oracle_pose_energy failed ({rc})")
    return out


def site_energy(case, xyz, site: int = 0) -> np.ndarray:
    """TriclinicSitePotential(case).evaluate(xyz, sigma_site, epsilon_site)."""
    cell, n, frac, sig, eps = _frame(case)
    xyz = _c(xyz)
    out = np.empty(len(xyz))
    rc = load().oracle_site_energy(_ptr(cell), n, _ptr(frac), _ptr(sig), _ptr(eps),
                                   float(case["guest_sigma"][site]),
                                   float(case["guest_epsilon"][site]), float(case["cutoff"]),
                                   len(xyz), _ptr(xyz), _ptr(out))
    if rc:
        raise RuntimeError(f"oracle_site_energy failed ({rc})")
    return out


def pair_counts(case, centers_frac, axes) -> np.ndarray:
    """In-cutoff (site, image) pairs per pose (the algorithmic unit of work)."""
    cell, n, frac, _, _ = _frame(case)
    centers, axes = _c(centers_frac), _c(axes)
    out = np.empty((len(centers), len(axes)), dtype=np.int64)
    rc = load().oracle_pair_counts(_ptr(cell), n, _ptr(frac), _ptr(_c(body_offsets(case))),
                                   float(case["cutoff"]), len(centers), _ptr(centers), len(axes),
                                   _ptr(axes), _ptr(out))
    if rc:
        raise RuntimeError(f"oracle_pair_counts failed ({rc})")
    return out


def pose_energy_grad(case, centers_cart, directors):
    """FP64 energy, dE/d(center) and dE/d(director) of poses (n, 3) + (n, 3)."""
    cell, n, frac, sig, eps = _frame(case)
    c, u = _c(centers_cart), _c(directors)
    m = len(c)
    e, gc, gu = np.empty(m), np.empty((m, 3)), np.empty((m, 3))
    rc = load().oracle_pose_energy_grad(_ptr(cell), n, _ptr(frac), _ptr(sig), _ptr(eps),
                                        float(case["guest_sigma"][0]),
                                        float(case["guest_epsilon"][0]),
                                        _ptr(_c(body_offsets(case))), float(case["cutoff"]), m,
                                        _ptr(c), _ptr(u), _ptr(e), _ptr(gc), _ptr(gu))
    if rc:
        raise RuntimeError(f"oracle_pose_energy_grad failed ({rc})")
    return e, gc, gu


def pair_lj(cell, site, atom_frac, sigma=3.5, epsilon=98., sigma_frame=3.4, epsilon_frame=50.,
            cutoff=5.5) -> float:
    """triclinic_pair.h:14-68 restated; ``cell`` is the row-vector cell."""
    cols = [_c(np.asarray(cell, dtype=float)[:, k]) for k in range(3)]
    return load().oracle_pair_lj(float(site[0]), float(site[1]), float(site[2]),
                                 float(atom_frac[0]), float(atom_frac[1]), float(atom_frac[2]),
                                 *(_ptr(col) for col in cols), float(epsilon), float(sigma),
                                 float(epsilon_frame), float(sigma_frame), float(cutoff))


def euler_pose_energy(case, poses) -> np.ndarray:
    """String pose energy (global.h:1071-1128); poses (n, 6) = frac a b c, Euler a b g (rad)."""
    cell, n, frac, sig, eps = _frame(case)
    poses = _c(poses)
    body = _c(case["guest_xyz"])
    out = np.empty(len(poses))
    rc = load().oracle_euler_pose_energy(_ptr(cell), n, _ptr(frac), _ptr(sig), _ptr(eps), 2,
                                         _ptr(body), _ptr(_c(case["guest_sigma"])),
                                         _ptr(_c(case["guest_epsilon"])), float(case["cutoff"]),
                                         len(poses), _ptr(poses), _ptr(out))
    if rc:
        raise RuntimeError(f"oracle_euler_pose_energy failed ({rc})")
    return out


def string_fd_gradient(case, poses, delta_frac=1e-4, delta_angle_rad=np.pi / 180,
                       rounding=1e-15) -> np.ndarray:
    """The reference String "forces" (global.h:1141-1325): for each pose the
    one-sided difference E(x + h e_k) - E(x) over (a, b, c, alpha, beta, gamma),
    NOT divided by h, truncated as floor(g / 1e-15) * 1e-15.  Returns (n, 6)."""
    poses = np.asarray(poses, dtype=float)
    shifted = np.repeat(poses[:, None, :], 7, axis=1)
    for k in range(6):
        shifted[:, k + 1, k] += delta_frac if k < 3 else delta_angle_rad
    energy = euler_pose_energy(case, shifted.reshape(-1, 6)).reshape(-1, 7)
    grad = energy[:, 1:] - energy[:, :1]
    return np.floor(grad / rounding) * rounding


# ---------------------------------------------------------------------------
# Restatement of the reference CPU driver (native.py / neighbor.py / physics.py)
# ---------------------------------------------------------------------------

class ReferenceDriver:
    """``NativeReusePotential`` restated: images and per-image coefficients as
    ``ReusePotential`` builds them, a cKDTree over the images, 512-center CSR
    batches, one ``evaluate_reused_neighbors`` call per batch."""

    def __init__(self, case: dict, library, batch_size: int = 512,
                 symbol: str = "evaluate_reused_neighbors"):
        from scipy.spatial import cKDTree
        sigma = np.asarray(case["guest_sigma"], dtype=float)
        epsilon = np.asarray(case["guest_epsilon"], dtype=float)
        if sigma[0] != sigma[1] or epsilon[0] != epsilon[1]:
            raise ValueError("exact neighbor reuse requires identical two-site LJ parameters")
        self.case = case
        self.offsets = _c(body_offsets(case))
        self.cutoff = float(case["cutoff"])
        self.radius = self.cutoff + float(np.abs(self.offsets).max())
        self.cell = np.asarray(case["cell"], dtype=float)
        inverse = np.linalg.inv(self.cell)
        spacing = 1 / np.linalg.norm(inverse, axis=0)
        reach = np.ceil(self.radius / spacing).astype(int) + 1
        shifts = np.array(list(itertools.product(*[range(-r, r + 1) for r in reach])), dtype=float)
        atoms = np.mod(case["frame_frac"], 1)
        self.images = _c((atoms[None] + shifts[:, None]).reshape(-1, 3) @ self.cell)
        fs = np.tile(case["frame_sigma"], len(shifts))
        fe = np.tile(case["frame_epsilon"], len(shifts))
        ms = (fs + sigma[0]) / 2
        me = np.sqrt(fe * epsilon[0])
        s6 = ms**6
        self.coeff12 = _c(4 * me * s6**2)
        self.coeff6 = _c(4 * me * s6)
        cut6 = (ms / self.cutoff)**6
        self.shift = _c(-4 * me * (cut6**2 - cut6))
        self.floor2 = _c((.1 * ms)**2)
        self.tree = cKDTree(self.images)
        self.batch_size = batch_size
        self.library = ctypes.CDLL(str(Path(library).resolve()))
        self.kernel = getattr(self.library, symbol)
        self.kernel.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_double] + [ctypes.c_void_p] * 11
        self.kernel.restype = ctypes.c_int
        self.query_seconds = 0.0
        self.compute_seconds = 0.0
        self.max_neighbors = 0

    def evaluate(self, centers_frac, axes) -> np.ndarray:
        centers = np.asarray(centers_frac, dtype=float)
        axes = np.asarray(axes, dtype=float)
        axes = _c(axes / np.linalg.norm(axes, axis=1, keepdims=True))
        cart = _c(np.mod(centers, 1) @ self.cell)
        out = np.empty((len(cart), len(axes)))
        for start in range(0, len(cart), self.batch_size):
            end = min(start + self.batch_size, len(cart))
            stamp = time.perf_counter()
            groups = self.tree.query_ball_point(cart[start:end], self.radius, workers=1)
            lengths = np.fromiter((len(g) for g in groups), dtype=np.int64, count=len(groups))
            starts = np.zeros(len(groups) + 1, dtype=np.int64)
            starts[1:] = np.cumsum(lengths)
            indices = (np.concatenate([np.asarray(g, dtype=np.int32) for g in groups])
                       if starts[-1] else np.empty(0, np.int32))
            self.max_neighbors = max(self.max_neighbors, int(lengths.max(initial=0)))
            self.query_seconds += time.perf_counter() - stamp
            stamp = time.perf_counter()
            block = _c(cart[start:end])
            view = out[start:end]
            rc = self.kernel(end - start, len(axes), len(self.images), self.cutoff**2,
                             _ptr(block), _ptr(axes), _ptr(self.images), _ptr(self.offsets),
                             _ptr(self.coeff12), _ptr(self.coeff6), _ptr(self.shift),
                             _ptr(self.floor2), _ptr(starts), _ptr(indices), _ptr(view))
            if rc:
                raise RuntimeError(f"native neighbor kernel failed with code {rc}")
            self.compute_seconds += time.perf_counter() - stamp
        if not np.isfinite(out).all():
            raise ValueError("nonfinite native Vext energy")
        return out


def reference_driver_class():
    """The reference's own ``NativeReusePotential`` (src/string_vext/native.py)
    when its package is installed in ``baseline/_ref``, else None."""
    if not (REF_PACKAGE / "string_vext" / "native.py").exists():
        return None
    import sys
    if str(REF_PACKAGE) not in sys.path:
        sys.path.append(str(REF_PACKAGE))
    from string_vext.native import NativeReusePotential
    return NativeReusePotential


def cpu_driver(case, library, symbol="evaluate_reused_neighbors"):
    """The reference CPU path's driver: the reference's own class when its
    package is installed and the symbol is the reference's, else the
    restatement above.  Returns (driver, which)."""
    cls = reference_driver_class() if symbol == "evaluate_reused_neighbors" else None
    if cls is not None:
        return cls(case, library), "reference driver (baseline/_ref)"
    return ReferenceDriver(case, library, symbol=symbol), "restated driver (oracle)"


def _shard_worker(args):
    case, library, centers, axes, symbol = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    driver, _ = cpu_driver(case, library, symbol)
    t0 = time.perf_counter()
    out = driver.evaluate(centers, axes)
    return out, time.perf_counter() - t0, driver.query_seconds, driver.compute_seconds


def reference_field_parallel(case, centers_frac, axes, library=REF_KERNEL, processes=None,
                             symbol="evaluate_reused_neighbors"):
    """The reference's multi-process mode (one driver per worker over disjoint
    center shards, as its ``--workers`` batch runners do).  Uses a ``spawn``
    pool.  Returns (energy (n_centers, n_axes), wall seconds including the
    pool start, processes, compute seconds = the slowest worker's
    neighbour-query + kernel time)."""
    import multiprocessing as mp
    processes = processes or max(1, len(os.sched_getaffinity(0)))
    shards = np.array_split(np.arange(len(centers_frac)), processes)
    jobs = [(case, str(library), np.asarray(centers_frac)[s], axes, symbol)
            for s in shards if len(s)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        parts = pool.map(_shard_worker, jobs)
    wall = time.perf_counter() - t0
    return (np.concatenate([p[0] for p in parts]), wall, len(jobs),
            max(p[1] for p in parts))
