"""Batched poses of many systems in one launch (vext_pose_batch_*): String
paths of several frameworks x guests, forward + adjoint, through the C ABI.

Checked against the FP64 oracle's analytic energy and gradient (mixed mode:
1e-4 K absolute where E <= 0, 1e-6 relative above, gradient 1e-5 relative
with a 1 K/A floor; FP64 mode: 1e-10 / 1e-9), against the single-system pose
entry, and for repeatability."""
import numpy as np
import pytest
import torch

from oracle import oracle
from string_vext_b200 import _lib, synth
from string_vext_b200.system import VextPoseBatch, VextSystem

pytestmark = pytest.mark.gpu


def quat_director(q):
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)], 1)


def workload(n_paths=8, masses=None):
    cases = synth.batch_frameworks(3) + [synth.small_field()]
    if masses is not None:   # unequal site masses: sites off-center, o_1 != -o_0
        cases = [dict(c, guest_mass=np.asarray(masses, dtype=float),
                      total_mass=float(sum(masses))) for c in cases]
    paths = synth.string_paths_batch(cases, n_paths=n_paths)
    # group the paths by system (the batch's layout)
    order = sorted(range(len(paths)), key=lambda p: paths[p][0])
    per_sys = [[] for _ in cases]
    for p in order:
        k, frac, quat = paths[p]
        per_sys[k].append((frac @ np.asarray(cases[k]["cell"], dtype=float), quat))
    centers, quats, counts = [], [], []
    for k in range(len(cases)):
        counts.append(sum(len(c) for c, _ in per_sys[k]))
        for c, q in per_sys[k]:
            centers.append(c)
            quats.append(q)
    return cases, counts, np.concatenate(centers), np.concatenate(quats)


def run_batch(systems, counts, centers, quats, mode):
    n = len(centers)
    dev = dict(dtype=torch.float64, device="cuda")
    c, q = torch.tensor(centers, **dev), torch.tensor(quats, **dev)
    e, gc = torch.empty(n, **dev), torch.empty((n, 3), **dev)
    gq, gu = torch.empty((n, 4), **dev), torch.empty((n, 3), **dev)
    batch = VextPoseBatch(systems, counts, mode=mode)
    batch.run(c, q, e, gc, gq, gu)
    batch.check()
    out = [t.cpu().numpy() for t in (e, gc, gq, gu)]
    batch.run(c, q, e, gc, gq, gu)
    batch.check()
    again = [t.cpu().numpy() for t in (e, gc, gq, gu)]
    for a, b in zip(out, again):
        np.testing.assert_array_equal(a, b)
    batch.close()
    return out


def oracle_refs(cases, counts, centers, quats):
    dirs = quat_director(quats)
    e, gc, gu = [], [], []
    start = 0
    for case, n in zip(cases, counts):
        if n:
            ee, cc, uu = oracle.pose_energy_grad(case, centers[start:start + n],
                                                 dirs[start:start + n])
            e.append(ee)
            gc.append(cc)
            gu.append(uu)
        start += n
    return np.concatenate(e), np.concatenate(gc), np.concatenate(gu)


def rel_rows(a, b, floor=1.0):
    return np.linalg.norm(a - b, axis=-1) / np.maximum(np.linalg.norm(b, axis=-1), floor)


@pytest.mark.parametrize("masses", [None, (15.0, 25.0)])
@pytest.mark.parametrize("mode", [_lib.VEXT_MODE_MIXED, _lib.VEXT_MODE_FP64])
def test_pose_batch_matches_oracle_and_single_entry(mode, masses):
    cases, counts, centers, quats = workload(masses=masses)
    systems = [VextSystem(c) for c in cases]
    e, gc, gq, gu = run_batch(systems, counts, centers, quats, mode)
    e_ref, gc_ref, gu_ref = oracle_refs(cases, counts, centers, quats)
    rel = np.abs(e - e_ref) / np.maximum(np.abs(e_ref), 1.0)
    if mode == _lib.VEXT_MODE_FP64:
        assert rel.max() < 1e-10
        assert rel_rows(gc, gc_ref).max() < 1e-9
        assert rel_rows(gu, gu_ref).max() < 1e-9
    else:
        neg = e_ref <= 0
        if neg.any():
            assert np.abs(e - e_ref)[neg].max() < 1e-4
        assert rel[~neg].max() < 1e-6
        assert rel_rows(gc, gc_ref).max() < 1e-5
        assert rel_rows(gu, gu_ref).max() < 1e-5
    # the single-system entry on the same poses
    start = 0
    for system, n in zip(systems, counts):
        if n:
            se, sgc, sgq, sgu = system.pose_energy_grad(centers[start:start + n],
                                                        quats[start:start + n], mode=mode)
            # each within the bar of FP64: the two mixed results within twice it
            tol = 1e-10 if mode == _lib.VEXT_MODE_FP64 else 2e-6
            np.testing.assert_allclose(e[start:start + n], se, rtol=tol,
                                       atol=1e-8 if tol < 1e-8 else 2e-4)
            assert rel_rows(gq[start:start + n], sgq).max() < (1e-9 if tol < 1e-8 else 1e-5)
        start += n
    for s in systems:
        s.close()


def test_pose_batch_rejects_bad_input():
    cases, counts, centers, quats = workload(n_paths=4)
    systems = [VextSystem(c) for c in cases]
    quats = quats.copy()
    quats[0] = 0.0
    with pytest.raises(_lib.VextError):
        run_batch(systems, counts, centers, quats, _lib.VEXT_MODE_MIXED)
    with pytest.raises(_lib.VextError):
        VextPoseBatch(systems, [-1] + counts[1:])
    for s in systems:
        s.close()
