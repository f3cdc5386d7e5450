"""Pose energies and the hand-written adjoint through the C ABI: against the
FP64 oracle's analytic gradient, FP64 central differences, and the
reference String solver's forward-difference forces (restated in the
oracle, global.h:1141-1325); the torch autograd Function."""
import numpy as np
import pytest
import torch

from oracle import oracle
from string_vext_b200 import _lib, synth
from string_vext_b200.autograd import pose_energy
from string_vext_b200.physics import body_offsets
from string_vext_b200.system import VextSystem

pytestmark = pytest.mark.gpu

FP64 = _lib.VEXT_MODE_FP64
MIXED = _lib.VEXT_MODE_MIXED


def director(q):
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)], 1)


def random_poses(case, n, seed):
    rng = np.random.default_rng(seed)
    frac = rng.random((n, 3))
    q = rng.normal(size=(n, 4))
    return frac @ case["cell"], q / np.linalg.norm(q, axis=1, keepdims=True)


@pytest.fixture(scope="module")
def small():
    case = synth.small_field()
    with VextSystem(case) as system:
        yield case, system


def test_fp64_energy_and_gradient_match_oracle(small):
    case, system = small
    c, q = random_poses(case, 200, 11)
    e, gc, gq, gu = system.pose_energy_grad(c, q, mode=FP64)
    re, rgc, rgu = oracle.pose_energy_grad(case, c, director(q))
    np.testing.assert_allclose(e, re, rtol=1e-10, atol=1e-8)
    scale = np.maximum(np.abs(rgc).max(axis=1, keepdims=True), 1.0)
    assert (np.abs(gc - rgc) / scale).max() < 1e-9
    assert (np.abs(gu - rgu) / np.maximum(np.abs(rgu).max(axis=1, keepdims=True), 1.0)).max() < 1e-9


def test_mixed_matches_fp64(small):
    case, system = small
    c, q = random_poses(case, 4096, 12)
    e64, gc64, gq64, _ = system.pose_energy_grad(c, q, mode=FP64)
    e, gc, gq, _ = system.pose_energy_grad(c, q, mode=MIXED)
    neg = e64 <= 0
    assert np.abs(e - e64)[neg].max() < 1e-4
    assert (np.abs(e - e64) / np.maximum(np.abs(e64), 1))[~neg].max() < 1e-6
    scale = np.maximum(np.abs(gc64).max(axis=1, keepdims=True), 1.0)
    assert (np.abs(gc - gc64) / scale).max() < 1e-5


def test_gradients_match_central_differences(small):
    """dE/dcenter and dE/dq (tangent) vs FP64 central differences,
    h = 1e-4 A and 1e-4 rad, on accessible poses."""
    case, system = small
    c, q = random_poses(case, 512, 13)
    e, gc, gq, _ = system.pose_energy_grad(c, q, mode=FP64)
    keep = e < 1e3
    c, q, gc, gq = c[keep][:64], q[keep][:64], gc[keep][:64], gq[keep][:64]
    h = 1e-4
    for k in range(3):
        d = np.zeros(3)
        d[k] = h
        ep, *_ = system.pose_energy_grad(c + d, q, mode=FP64, grad=False)
        em, *_ = system.pose_energy_grad(c - d, q, mode=FP64, grad=False)
        fd = (ep - em) / (2 * h)
        np.testing.assert_allclose(gc[:, k], fd, rtol=1e-5, atol=1e-5 * np.abs(gc).max())
    # rotate by a small angle t about lab axis e_k: q(t) = exp(t e_k / 2) q,
    # a tangent direction with dq/dt = (0, e_k / 2) q at t = 0
    def qmul(a, b):
        w = a[..., 0] * b[..., 0] - (a[..., 1:] * b[..., 1:]).sum(-1)
        v = (a[..., :1] * b[..., 1:] + b[..., :1] * a[..., 1:]
             + np.cross(a[..., 1:], b[..., 1:]))
        return np.concatenate([w[..., None], v], -1)

    for k in range(3):
        axis = np.zeros(3)
        axis[k] = 1.0
        rot = lambda t: qmul(np.r_[np.cos(t / 2), np.sin(t / 2) * axis][None], q)
        ep, *_ = system.pose_energy_grad(c, rot(h), mode=FP64, grad=False)
        em, *_ = system.pose_energy_grad(c, rot(-h), mode=FP64, grad=False)
        fd = (ep - em) / (2 * h)
        dq = qmul(np.r_[0.0, axis / 2][None], q)
        np.testing.assert_allclose((gq * dq).sum(1), fd, rtol=1e-5, atol=1e-5 * np.abs(fd).max())


def test_against_reference_string_forces(small):
    """The reference's String 'forces' are one-sided differences over
    (frac a, b, c, Euler alpha, beta, gamma), not divided by the step.  With
    small steps they equal step x the analytic gradient in those coordinates."""
    case, system = small
    rng = np.random.default_rng(14)
    poses = np.column_stack([rng.random((3000, 3)), rng.uniform(-np.pi, np.pi, (3000, 3))])
    # String images are accessible poses; keep those (E < 1e4 K)
    poses = poses[oracle.euler_pose_energy(case, poses) < 1e4][:24]
    assert len(poses) >= 12
    hf, ha = 1e-7, 1e-7
    ref = oracle.string_fd_gradient(case, poses, delta_frac=hf, delta_angle_rad=ha,
                                    rounding=1e-15)
    a, b, g = poses[:, 3], poses[:, 4], poses[:, 5]
    u = np.stack([np.cos(g) * np.cos(b), np.sin(g) * np.cos(b), -np.sin(b)], 1)
    # quaternion of R = Rz(g) Ry(b) Rx(a)
    ca, sa, cb, sb, cg, sg = (np.cos(a / 2), np.sin(a / 2), np.cos(b / 2), np.sin(b / 2),
                              np.cos(g / 2), np.sin(g / 2))
    quat = np.stack([cg * cb * ca + sg * sb * sa, cg * cb * sa - sg * sb * ca,
                     cg * sb * ca + sg * cb * sa, sg * cb * ca - cg * sb * sa], 1)
    np.testing.assert_allclose(director(quat), u, atol=1e-12)
    e, gc, _, gu = system.pose_energy_grad(poses[:, :3] @ case["cell"], quat, mode=FP64)
    np.testing.assert_allclose(e, oracle.euler_pose_energy(case, poses), rtol=1e-10, atol=1e-8)
    g_frac = gc @ case["cell"].T
    du_db = np.stack([-np.cos(g) * np.sin(b), -np.sin(g) * np.sin(b), -np.cos(b)], 1)
    du_dg = np.stack([-np.sin(g) * np.cos(b), np.cos(g) * np.cos(b), np.zeros_like(b)], 1)
    analytic = np.column_stack([g_frac * hf, np.zeros(len(a)), (gu * du_db).sum(1) * ha,
                                (gu * du_dg).sum(1) * ha])
    scale = np.maximum(np.abs(analytic).max(axis=1, keepdims=True), 1e-9)
    assert (np.abs(analytic - ref) / scale).max() < 1e-4


def test_autograd_function(small):
    case, system = small
    c, q = random_poses(case, 256, 15)
    ct = torch.tensor(c, device="cuda", requires_grad=True)
    qt = torch.tensor(q, device="cuda", requires_grad=True)
    e = pose_energy(system, ct, qt, _lib.VEXT_MODE_FP64)
    weights = torch.linspace(0.5, 1.5, len(c), device="cuda", dtype=torch.float64)
    (e * weights).sum().backward()
    e_np, gc, gq, _ = system.pose_energy_grad(c, q, mode=FP64)
    np.testing.assert_allclose(e.detach().cpu().numpy(), e_np, rtol=0, atol=0)
    w = weights.cpu().numpy()[:, None]
    np.testing.assert_allclose(ct.grad.cpu().numpy(), w * gc, rtol=1e-14, atol=0)
    np.testing.assert_allclose(qt.grad.cpu().numpy(), w * gq, rtol=1e-14, atol=0)


def test_string_path_and_random_batch():
    case, pf, pq, bf, bq = synth.string_path()
    with VextSystem(case) as system:
        for frac, quat in ((pf, pq), (bf[:8192], bq[:8192])):
            cart = frac @ case["cell"]
            e64, gc64, *_ = system.pose_energy_grad(cart, quat, mode=FP64)
            e, gc, *_ = system.pose_energy_grad(cart, quat, mode=MIXED)
            neg = e64 <= 0
            assert np.abs(e - e64)[neg].max(initial=0) < 1e-4
            assert (np.abs(e - e64) / np.maximum(np.abs(e64), 1))[~neg].max(initial=0) < 1e-6
            ref = oracle.pose_energy_grad(case, cart[:64], director(quat[:64]))[0]
            np.testing.assert_allclose(e64[:64], ref, rtol=1e-10, atol=1e-8)


@pytest.mark.parametrize("n", [1, 7, 301, 1000])
def test_small_batches_of_any_size(small, n):
    """Small batches take the kernel that spreads each pose's bin list over one
    to eight warps (8 for n <= 296, 4 for n = 301 with one idle warp group in
    the last CTA, 2 for n = 1000): mixed within the bar of the FP64 oracle,
    FP64 to 1e-10."""
    case, system = small
    c, q = random_poses(case, n, 100 + n)
    re, rgc, rgu = oracle.pose_energy_grad(case, c, director(q))
    e, gc, gq, gu = system.pose_energy_grad(c, q, mode=FP64)
    np.testing.assert_allclose(e, re, rtol=1e-10, atol=1e-8)
    scale = np.maximum(np.abs(rgc).max(axis=1, keepdims=True), 1.0)
    assert (np.abs(gc - rgc) / scale).max() < 1e-9
    e, gc, gq, gu = system.pose_energy_grad(c, q, mode=MIXED)
    neg = re <= 0
    if neg.any():
        assert np.abs(e - re)[neg].max() < 1e-4
    assert (np.abs(e - re) / np.maximum(np.abs(re), 1))[~neg].max() < 1e-6
    assert (np.abs(gc - rgc) / scale).max() < 1e-5
    scale_u = np.maximum(np.abs(rgu).max(axis=1, keepdims=True), 1.0)
    assert (np.abs(gu - rgu) / scale_u).max() < 1e-5


def lone_atom_case(length):
    """One framework atom in a cubic cell wider than twice the cutoff: a site
    sees at most one image of it, so a pose's forces are those of one or two
    pairs (about 0.06 K/A at the cutoff)."""
    return synth.make_case([length] * 3, [90.0] * 3, np.array([[0.5, 0.5, 0.5]]), [3.4], [60.0],
                           synth.GUEST_A, 12.0)


def border_poses(case, n, seed):
    """Poses whose site 0 sits 1e-9 relative inside or outside the cutoff of
    the lone atom (|d2 - rc^2| ~ 3e-7 A^2: far below the FP32 error of d2, far
    above FP64 rounding), random directors."""
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    u = director(q)
    off0 = body_offsets(case)[0]
    atom = case["frame_frac"][0] @ case["cell"]
    w = rng.normal(size=(n, 3))
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    scale = np.where(np.arange(n) % 2 == 0, 1.0 - 1e-9, 1.0 + 1e-9)
    site0 = atom + (case["cutoff"] * scale)[:, None] * w
    return site0 - off0 * u, q


@pytest.mark.parametrize("length,n_random", [(40.0, 0), (25.0, 2_600_000)])
def test_pairs_at_the_cutoff_are_decided_in_fp64(length, n_random):
    """A site-atom pair at the cutoff (to 1e-9) must be counted as the FP64
    test counts it: a pair decided the other way would move the pose's
    gradient by the force jump at rc (about 0.06 K/A, here the whole force).
    Mixed against FP64 mode within 1e-6 (K, K/A, K per quaternion unit) on
    such poses, through the warp-per-pose path (64 poses) and the binned pose
    kernel (2.6 M random poses around them, more than 64 per bin)."""
    case = lone_atom_case(length)
    cb, qb = border_poses(case, 64, 17)
    if n_random:
        cr, qr = random_poses(case, n_random, 18)
        cb, qb = np.concatenate([cb, cr]), np.concatenate([qb, qr])
    with VextSystem(case) as system:
        e, gc, gq, _ = system.pose_energy_grad(cb, qb, mode=MIXED)
        e64, gc64, gq64, _ = system.pose_energy_grad(cb[:64], qb[:64], mode=FP64)
    assert np.abs(gc64).max() > 0.01          # the poses do feel the border pairs
    assert np.abs(e[:64] - e64).max() < 1e-6
    assert np.abs(gc[:64] - gc64).max() < 1e-6
    assert np.abs(gq[:64] - gq64).max() < 1e-6


def test_asymmetric_guest_pose_path():
    """Unequal site masses put the sites off-center (o_1 != -o_0); the pose
    kernels carry each site's offset: FP64 mode against the oracle, mixed
    against FP64 mode within the bar, on random poses (warp-per-pose path)."""
    case = dict(synth.small_field())
    case["guest_mass"] = np.array([15.0, 25.0])
    case["total_mass"] = 40.0
    cart, q = random_poses(case, 512, 23)
    with VextSystem(case) as system:
        e, gc, gq, _ = system.pose_energy_grad(cart, q, mode=MIXED)
        e64, gc64, gq64, gu64 = system.pose_energy_grad(cart, q, mode=FP64)
    re, rgc, rgu = oracle.pose_energy_grad(case, cart, director(q))
    np.testing.assert_allclose(e64, re, rtol=1e-10, atol=1e-8)
    assert (np.abs(gc64 - rgc) / np.maximum(np.abs(rgc).max(axis=1, keepdims=True), 1.0)).max() < 1e-9
    neg = e64 <= 0
    assert np.abs(e - e64)[neg].max(initial=0) < 1e-4
    assert (np.abs(e - e64) / np.maximum(np.abs(e64), 1))[~neg].max() < 1e-6
    scale = np.maximum(np.linalg.norm(gc64, axis=1), 1.0)
    assert (np.linalg.norm(gc - gc64, axis=1) / scale).max() < 1e-5
