"""Forward + adjoint over the field poses (energy, dE/d(center), tangent
dE/d(director) at every grid center x director) through the C ABI, against
the FP64 oracle's analytic gradient and against central finite differences of
the FP64 oracle energy.

Tolerances: the plain FP64 kernel agrees with the oracle to 1e-10 relative
(energy, floor 1 K) and 1e-9 relative (gradient norm, floor 1 K/A); the mixed
kernel keeps the energy bar on its FP64 energy output (1e-4 K absolute where
E <= 0, 1e-6 relative above; the float32 output is its rounding) and its
gradient agrees with the oracle and with central differences (h = 1e-4 A,
1e-4 rad) to 1e-5 relative.
"""
import numpy as np
import pytest
import torch

from oracle import oracle
from string_vext_b200 import _lib, synth
from string_vext_b200.orientation import normalized_directors, regular_pose_grid
from string_vext_b200.system import VextBatch, VextSystem

pytestmark = pytest.mark.gpu

FP64 = _lib.VEXT_MODE_FP64
MIXED = _lib.VEXT_MODE_MIXED


def field_poses(case, size, n_axes=64):
    """Cartesian centers and directors of every pose in [O][S^3] order."""
    frac, axes = regular_pose_grid(size, n_axes)
    axes = normalized_directors(axes)
    cart = frac @ np.asarray(case["cell"], dtype=float)
    centers = np.broadcast_to(cart[None], (n_axes,) + cart.shape).reshape(-1, 3)
    dirs = np.broadcast_to(axes[:, None, :], (n_axes, len(cart), 3)).reshape(-1, 3)
    return axes, np.ascontiguousarray(centers), np.ascontiguousarray(dirs)


def oracle_field_adjoint(case, size, n_axes=64):
    axes, centers, dirs = field_poses(case, size, n_axes)
    e, gc, gu = oracle.pose_energy_grad(case, centers, dirs)
    gu_t = gu - (gu * dirs).sum(1)[:, None] * dirs
    shape = (n_axes, size, size, size)
    return axes, e.reshape(shape), np.concatenate([gc, gu_t], 1).reshape(shape + (6,))


def grad_rel(g, ref):
    """Per-pose relative error of the 6-vector gradient (floor 1 K/A)."""
    diff = np.linalg.norm(g - ref, axis=-1)
    return diff / np.maximum(np.linalg.norm(ref, axis=-1), 1.0)


def run_device(system, size, axes, mode, energy64=False, grad64=False):
    n = len(axes)
    shape = (n, size, size, size)
    e = torch.empty(shape, dtype=torch.float32, device="cuda")
    g = torch.empty(shape + (6,), dtype=torch.float32, device="cuda")
    e64 = torch.empty(shape, dtype=torch.float64, device="cuda") if energy64 else None
    g64 = torch.empty(shape + (6,), dtype=torch.float64, device="cuda") if grad64 else None
    system.field_adjoint_device(size, axes, e, g, e64, g64, mode=mode)
    torch.cuda.synchronize()
    out = [e.cpu().numpy(), g.cpu().numpy()]
    out += [t.cpu().numpy() for t in (e64, g64) if t is not None]
    return out


@pytest.mark.parametrize("maker,size", [(synth.small_field, 4), (synth.full_field, 3),
                                        (synth.skewed_field, 3)])
def test_fp64_and_mixed_adjoint_match_oracle(maker, size):
    case = maker()
    axes, e_ref, g_ref = oracle_field_adjoint(case, size)
    with VextSystem(case) as system:
        e32, g32, e64, g64 = run_device(system, size, axes, FP64, energy64=True, grad64=True)
        me, mg, me64 = run_device(system, size, axes, MIXED, energy64=True)
    assert (np.abs(e64 - e_ref) / np.maximum(np.abs(e_ref), 1)).max() < 1e-10
    assert grad_rel(g64, g_ref).max() < 1e-9
    np.testing.assert_array_equal(e32, e64.astype(np.float32))
    np.testing.assert_array_equal(g32, g64.astype(np.float32))
    np.testing.assert_array_equal(me, me64.astype(np.float32))
    neg = e_ref <= 0
    if neg.any():
        assert np.abs(me64 - e_ref)[neg].max() < 1e-4
    if (~neg).any():
        assert (np.abs(me64 - e_ref) / np.maximum(np.abs(e_ref), 1))[~neg].max() < 1e-6
    assert grad_rel(mg.astype(np.float64), g_ref).max() < 1e-5


def test_mixed_gradient_matches_central_differences():
    """dE/dc and the tangent dE/du of accessible poses (E < 0) against central
    differences of the FP64 oracle energy, h = 1e-4 A and 1e-4 rad."""
    case = synth.small_field()
    size = 6
    axes, centers, dirs = field_poses(case, size)
    with VextSystem(case) as system:
        me, mg = run_device(system, size, axes, MIXED)
    e = me.reshape(-1)
    g = mg.reshape(-1, 6).astype(np.float64)
    pick = np.flatnonzero(e < 0)
    assert len(pick) >= 32
    pick = pick[np.linspace(0, len(pick) - 1, 32).astype(int)]
    c, u = centers[pick], dirs[pick]
    h = 1e-4
    fd = np.zeros((len(pick), 6))
    for k in range(3):
        step = np.zeros(3)
        step[k] = h
        ep, _, _ = oracle.pose_energy_grad(case, c + step, u)
        em, _, _ = oracle.pose_energy_grad(case, c - step, u)
        fd[:, k] = (ep - em) / (2 * h)
    # tangent basis e1, e2 normal to u; rotate u by +-h about each
    ref = np.where(np.abs(u[:, :1]) < 0.9, [[1.0, 0, 0]], [[0, 1.0, 0]])
    e1 = np.cross(u, ref)
    e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
    e2 = np.cross(u, e1)
    for basis in (e1, e2):
        up = np.cos(h) * u + np.sin(h) * basis
        um = np.cos(h) * u - np.sin(h) * basis
        ep, _, _ = oracle.pose_energy_grad(case, c, up)
        em, _, _ = oracle.pose_energy_grad(case, c, um)
        d_fd = (ep - em) / (2 * h)
        d_an = (g[pick, 3:] * basis).sum(1)
        scale = np.maximum(np.linalg.norm(g[pick, 3:], axis=1), 1.0)
        assert (np.abs(d_an - d_fd) / scale).max() < 1e-5
    gc = g[pick, :3]
    scale = np.maximum(np.linalg.norm(fd[:, :3], axis=1), 1.0)
    assert (np.linalg.norm(gc - fd[:, :3], axis=1) / scale).max() < 1e-5


def test_adjoint_batch_matches_single_fields_and_host_entry():
    cases = synth.batch_frameworks(2) + [synth.small_field()]
    size = 5
    _, axes = regular_pose_grid(size, 64)
    axes = normalized_directors(axes)
    systems = [VextSystem(c) for c in cases]
    shape = (64, size, size, size)
    outs = [torch.full(shape, -1.0, dtype=torch.float32, device="cuda") for _ in systems]
    grads = [torch.full(shape + (6,), -1.0, dtype=torch.float32, device="cuda")
             for _ in systems]
    batch = VextBatch(systems, size, axes, outs, gradients=grads)
    assert batch.info()["adjoint"]
    for _ in range(2):
        batch.run()
        batch.check()
        torch.cuda.synchronize()
        for k, (system, out, grad) in enumerate(zip(systems, outs, grads)):
            e, g = system.field_adjoint(size, axes)
            de, dg = run_device(system, size, axes, MIXED)
            np.testing.assert_array_equal(de, e)
            np.testing.assert_array_equal(dg, g)
            if k >= 4 or k % 2 == 0:    # the owner of its framework's shared lists
                np.testing.assert_array_equal(out.cpu().numpy(), e)
                np.testing.assert_array_equal(grad.cpu().numpy(), g)
            else:                       # guest B on guest A's lists: within the bar
                got, ge = out.cpu().numpy().astype(np.float64), e.astype(np.float64)
                assert (np.abs(got - ge) <= 2e-4 + 2e-6 * np.abs(ge)).all()
                gg, gs = grad.cpu().numpy().astype(np.float64), g.astype(np.float64)
                rel = (np.linalg.norm(gg - gs, axis=-1)
                       / np.maximum(np.linalg.norm(gs, axis=-1), 1.0))
                assert rel.max() < 2e-5
    batch.close()
    for s in systems:
        s.close()


def test_adjoint_rejects_bad_arguments():
    case = synth.small_field()
    _, axes = regular_pose_grid(4, 64)
    axes = normalized_directors(axes)
    with VextSystem(case) as system:
        e = torch.empty((64, 4, 4, 4), dtype=torch.float32, device="cuda")
        g64 = torch.empty((64, 4, 4, 4, 6), dtype=torch.float64, device="cuda")
        with pytest.raises(_lib.VextError):
            system.field_adjoint_device(4, axes, e, None)          # mixed needs both outputs
        g = torch.empty((64, 4, 4, 4, 6), dtype=torch.float32, device="cuda")
        with pytest.raises(_lib.VextError):
            system.field_adjoint_device(4, axes, e, g, None, g64)   # FP64 gradient: FP64 modes
        bad = axes.copy()
        bad[0, 0] = np.nan
        with pytest.raises(_lib.VextError):
            system.field_adjoint_device(4, bad, e, g)


@pytest.mark.parametrize("maker,size", [(synth.skewed_field, 5), (synth.small_field, 6)])
def test_every_batch_shape_gives_identical_results(maker, size):
    """Each CTA shape the autotuner may pick (pinned with batch_shape) does the
    same per-director arithmetic in the same order: forward and forward +
    adjoint outputs are bit-identical across the shapes of a kernel table
    (forward + adjoint: 8-center regions by default, 16-center regions with
    centers_per_region=16; the two tables' lists differ, so do their bits)."""
    case = maker()
    _, axes = regular_pose_grid(size, 64)
    axes = normalized_directors(axes)
    shape = (64, size, size, size)
    with VextSystem(case) as system:
        for cb, min_shapes in ((0, 2), (16, 5)):
            e = torch.empty(shape, dtype=torch.float32, device="cuda")
            g = torch.empty(shape + (6,), dtype=torch.float32, device="cuda")
            system.field_adjoint_device(size, axes, e, g, centers_per_region=cb)
            torch.cuda.synchronize()
            ref_e, ref_g = e.cpu().numpy(), g.cpu().numpy()
            probe = VextBatch([system], size, axes,
                              [torch.empty(shape, dtype=torch.float32, device="cuda")],
                              gradients=[torch.empty(shape + (6,), dtype=torch.float32,
                                                     device="cuda")],
                              centers_per_region=cb)
            n_adj = len({t["shape"] for t in probe.tuning()})
            probe.close()
            assert n_adj >= min_shapes
            for k in range(1, n_adj + 1):
                e = torch.empty(shape, dtype=torch.float32, device="cuda")
                g = torch.empty(shape + (6,), dtype=torch.float32, device="cuda")
                system.field_adjoint_device(size, axes, e, g, batch_shape=k,
                                            centers_per_region=cb)
                torch.cuda.synchronize()
                np.testing.assert_array_equal(e.cpu().numpy(), ref_e)
                np.testing.assert_array_equal(g.cpu().numpy(), ref_g)
        fwd_ref = None
        for k in range(1, 3):
            out = torch.empty(shape, dtype=torch.float32, device="cuda")
            b = VextBatch([system], size, axes, [out], batch_shape=k)
            assert len(b.tuning()) == 1
            b.run()
            b.check()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            if fwd_ref is None:
                fwd_ref = got
            np.testing.assert_array_equal(got, fwd_ref)
            b.close()
        with pytest.raises(_lib.VextError):
            VextBatch([system], size, axes,
                      [torch.empty(shape, dtype=torch.float32, device="cuda")], batch_shape=99)


@pytest.mark.parametrize("size,n_axes", [(1, 7), (3, 33), (2, 40), (5, 1)])
def test_ragged_grids_and_director_counts(size, n_axes):
    """Director counts that are not multiples of the 32-director block (one
    more than a block: the host entry's split), a one-point grid, a single
    director: device and host entries agree bit for bit and match the oracle."""
    case = synth.small_field()
    rng = np.random.default_rng(size * 100 + n_axes)
    axes = normalized_directors(rng.normal(size=(n_axes, 3)))
    frac = (np.arange(size) + .5) / size
    grid = np.stack(np.meshgrid(frac, frac, frac, indexing="ij"), -1).reshape(-1, 3)
    cart = grid @ np.asarray(case["cell"], dtype=float)
    centers = np.ascontiguousarray(
        np.broadcast_to(cart[None], (n_axes,) + cart.shape).reshape(-1, 3))
    dirs = np.ascontiguousarray(
        np.broadcast_to(axes[:, None, :], (n_axes, len(cart), 3)).reshape(-1, 3))
    e_ref, gc, gu = oracle.pose_energy_grad(case, centers, dirs)
    gu = gu - (gu * dirs).sum(1)[:, None] * dirs
    g_ref = np.concatenate([gc, gu], 1)
    with VextSystem(case) as system:
        de, dg, de64 = run_device(system, size, axes, MIXED, energy64=True)
        he, hg = system.field_adjoint(size, axes)
    np.testing.assert_array_equal(he, de)
    np.testing.assert_array_equal(hg, dg)
    e = de64.reshape(-1)
    neg = e_ref <= 0
    if neg.any():
        assert np.abs(e - e_ref)[neg].max() < 1e-4
    assert (np.abs(e - e_ref) / np.maximum(np.abs(e_ref), 1))[~neg].max() < 1e-6
    assert grad_rel(dg.reshape(-1, 6).astype(np.float64), g_ref).max() < 1e-5


def test_host_entry_into_page_locked_buffers():
    """vext_field_adjoint with page-locked host outputs (the kernels write the
    float32 results straight into them) gives the same bits as with pageable
    outputs (staged copies) and as the device entry, including slices inside
    a larger page-locked allocation, whose neighbouring words stay untouched,
    and when calls switch between the two kinds of buffer."""
    import ctypes
    case = synth.small_field()
    size, n_axes = 6, 64
    _, axes = regular_pose_grid(size, n_axes)
    axes = normalized_directors(axes)
    shape = (n_axes, size, size, size)
    n = int(np.prod(shape))
    lib = _lib.load()
    opt = _lib.options()

    def host_call(system, e, g):
        _lib.check(lib.vext_field_adjoint(system.handle, size, n_axes, _lib.ptr(axes),
                                          ctypes.byref(opt), _lib.ptr(e), _lib.ptr(g)))

    with VextSystem(case) as system:
        ref_e, ref_g = run_device(system, size, axes, MIXED)
        for _ in range(2):
            pe = torch.full(shape, -7.0, dtype=torch.float32, pin_memory=True)
            pg = torch.full(shape + (6,), -7.0, dtype=torch.float32, pin_memory=True)
            host_call(system, pe, pg)
            np.testing.assert_array_equal(pe.numpy(), ref_e)
            np.testing.assert_array_equal(pg.numpy(), ref_g)
            e, g = system.field_adjoint(size, axes)      # pageable numpy outputs
            np.testing.assert_array_equal(e, ref_e)
            np.testing.assert_array_equal(g, ref_g)
            e, g = system.field_adjoint(size, axes, pinned=True)
            np.testing.assert_array_equal(e, ref_e)
            np.testing.assert_array_equal(g, ref_g)
        pad = 16
        be = torch.full((n + 2 * pad,), -7.0, dtype=torch.float32, pin_memory=True)
        bg = torch.full((6 * n + 2 * pad,), -7.0, dtype=torch.float32, pin_memory=True)
        se, sg = be[pad:pad + n], bg[pad:pad + 6 * n]
        host_call(system, se, sg)
        np.testing.assert_array_equal(se.numpy().reshape(shape), ref_e)
        np.testing.assert_array_equal(sg.numpy().reshape(shape + (6,)), ref_g)
        for big in (be, bg):
            assert (big[:pad] == -7.0).all() and (big[-pad:] == -7.0).all()


@pytest.mark.parametrize("mode", [FP64, _lib.VEXT_MODE_FP64_PLAIN])
def test_host_entry_fp64_modes(mode):
    """The host entry in the FP64 modes (staged copies) returns the device
    entry's float32 energy and gradient bit for bit."""
    case = synth.skewed_field()
    size = 5
    _, axes = regular_pose_grid(size, 64)
    axes = normalized_directors(axes)
    with VextSystem(case) as system:
        ref_e, ref_g = run_device(system, size, axes, mode)
        e, g = system.field_adjoint(size, axes, mode=mode)
        np.testing.assert_array_equal(e, ref_e)
        np.testing.assert_array_equal(g, ref_g)


def test_director_reversal_at_full_size():
    """Two identical sites at +-o: reversing every director swaps the sites, so
    on the full 60^3 x 64 field the energy and dE/dcenter are unchanged and the
    tangent dE/du changes sign, within the mixed bar of each result (both
    carry their own FP32 rounding: twice the bar)."""
    case = synth.full_field()
    size = 60
    _, axes = regular_pose_grid(size, 64)
    axes = normalized_directors(axes)
    shape = (64, size, size, size)
    with VextSystem(case) as system:
        results = []
        for a in (axes, -axes):
            e = torch.empty(shape, dtype=torch.float32, device="cuda")
            g = torch.empty(shape + (6,), dtype=torch.float32, device="cuda")
            e64 = torch.empty(shape, dtype=torch.float64, device="cuda")
            system.field_adjoint_device(size, np.ascontiguousarray(a), e, g, e64)
            torch.cuda.synchronize()
            results.append((e64, g))
        (ea, ga), (eb, gb) = results
        rel = ((ea - eb).abs() / ea.abs().clamp(min=1.0)).max().item()
        assert rel < 2e-6, rel
        scale = ga[..., :3].norm(dim=-1).clamp(min=1.0)
        assert ((ga[..., :3] - gb[..., :3]).norm(dim=-1) / scale).max().item() < 2e-5
        scale = ga[..., 3:].norm(dim=-1).clamp(min=1.0)
        assert ((ga[..., 3:] + gb[..., 3:]).norm(dim=-1) / scale).max().item() < 2e-5


def test_batch_frameworks_gradients_within_bar_for_every_pose():
    """The first 24 systems of the batched workload (12 seeded frameworks x
    both guests, uneven cells and atom counts), 12^3 x 64 poses each (2.65 M
    poses) through one forward + adjoint batch: every pose's gradient within
    1e-5 (norm relative to max(|grad E|, 1 K/A)) of the plain FP64 adjoint,
    energies within the bar.  A shell pair within FP32 rounding of the cutoff
    would move a gradient by the force jump at rc (about 0.05 K/A); such
    poses are re-evaluated in FP64, so no pose may exceed the bar."""
    cases = synth.batch_frameworks(12)
    size = 12
    _, axes = regular_pose_grid(size, 64)
    axes = normalized_directors(axes)
    systems = [VextSystem(c) for c in cases]
    shape = (64, size, size, size)
    outs = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in systems]
    grads = [torch.empty(shape + (6,), dtype=torch.float32, device="cuda") for _ in systems]
    batch = VextBatch(systems, size, axes, outs, gradients=grads)
    batch.run()
    batch.check()
    torch.cuda.synchronize()
    worst = 0.0
    for system, out, grad in zip(systems, outs, grads):
        e64 = torch.empty(shape, dtype=torch.float64, device="cuda")
        g64 = torch.empty(shape + (6,), dtype=torch.float64, device="cuda")
        system.field_adjoint_device(size, axes, None, None, e64, g64,
                                    mode=_lib.VEXT_MODE_FP64_PLAIN)
        torch.cuda.synchronize()
        ex, gx = e64.cpu().numpy(), g64.cpu().numpy()
        got = out.cpu().numpy().astype(np.float64)
        # float32 storage: compare the energies at float32 resolution
        assert (np.abs(got - ex) <= 1e-4 + 1.2e-7 * np.abs(ex)).all()
        gm = grad.cpu().numpy().astype(np.float64)
        grel = np.linalg.norm(gm - gx, axis=-1) / np.maximum(np.linalg.norm(gx, axis=-1), 1.0)
        worst = max(worst, float(grel.max()))
    batch.close()
    for s in systems:
        s.close()
    assert worst < 1e-5, f"worst gradient error {worst}"


def test_border_repair_matches_full_fp64_refinement():
    """Poses with a shell pair within 1.25e-4 A^2 of the cutoff get their shell
    pairs re-tested (the far kernel's FP32 decision recomputed bit for bit
    against the FP64 one, misjudged pairs swapped in or out in FP64).  The
    same batch with those poses wholly re-evaluated in FP64 (variant 4096)
    flags the same poses, and both results agree within FP32 resolution:
    energy at float32 storage, gradient 1e-6 relative.  Without the border
    test (variant 1024) only refinement-band poses are flagged."""
    cases = synth.batch_frameworks(4)
    size = 12
    _, axes = regular_pose_grid(size, 64)
    axes = normalized_directors(axes)
    systems = [VextSystem(c) for c in cases]
    shape = (64, size, size, size)
    results = {}
    for label, variant in (("repair", 0), ("full", 4096), ("none", 1024)):
        outs = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in systems]
        grads = [torch.empty(shape + (6,), dtype=torch.float32, device="cuda") for _ in systems]
        batch = VextBatch(systems, size, axes, outs, gradients=grads, variant=variant)
        batch.run()
        batch.check()
        refined = batch.refined()
        batch.close()
        results[label] = (refined, [o.cpu().numpy().astype(np.float64) for o in outs],
                          [g.cpu().numpy().astype(np.float64) for g in grads])
    for s in systems:
        s.close()
    n_rep, e_rep, g_rep = results["repair"]
    n_full, e_full, g_full = results["full"]
    assert n_rep == n_full > results["none"][0]   # "none": refinement-band poses only
    for a, b in zip(e_rep, e_full):
        assert (np.abs(a - b) <= 2e-4 + 2.4e-7 * np.abs(b)).all()
    for a, b in zip(g_rep, g_full):
        rel = np.linalg.norm(a - b, axis=-1) / np.maximum(np.linalg.norm(b, axis=-1), 1.0)
        assert rel.max() < 1e-6


def test_asymmetric_guest_takes_the_per_site_kernels():
    """Two identical sites of unequal mass sit off-center (o_1 != -o_0): the
    batch then runs the kernels that test the cutoff border per site and keep
    both sites' terms (the symmetric shortcuts do not apply).  Energies and
    gradients of every pose (small_field and a batch framework, 12^3 x 64)
    within the bar of the plain FP64 adjoint."""
    for case in (synth.small_field(), synth.batch_frameworks(1)[0]):
        case = dict(case)
        case["guest_mass"] = np.array([15.0, 25.0])
        case["total_mass"] = 40.0
        size = 12
        _, axes = regular_pose_grid(size, 64)
        axes = normalized_directors(axes)
        shape = (64, size, size, size)
        with VextSystem(case) as system:
            off = system.offsets
            assert off[0] != -off[1]
            out = torch.empty(shape, dtype=torch.float32, device="cuda")
            grad = torch.empty(shape + (6,), dtype=torch.float32, device="cuda")
            batch = VextBatch([system], size, axes, [out], gradients=[grad])
            assert "border/site" in batch.info()["cta_shape"]
            batch.run()
            batch.check()
            batch.close()
            e64 = torch.empty(shape, dtype=torch.float64, device="cuda")
            g64 = torch.empty(shape + (6,), dtype=torch.float64, device="cuda")
            system.field_adjoint_device(size, axes, None, None, e64, g64,
                                        mode=_lib.VEXT_MODE_FP64_PLAIN)
            torch.cuda.synchronize()
        ex, gx = e64.cpu().numpy(), g64.cpu().numpy()
        got = out.cpu().numpy().astype(np.float64)
        assert (np.abs(got - ex) <= 1e-4 + 1.2e-7 * np.abs(ex)).all()
        gm = grad.cpu().numpy().astype(np.float64)
        grel = np.linalg.norm(gm - gx, axis=-1) / np.maximum(np.linalg.norm(gx, axis=-1), 1.0)
        assert grel.max() < 1e-5


def test_outer_shell_single_site_pass_matches_two_site_pass():
    """Outer shell entries (beyond rc + the region radius from the region
    origin) can have only a director's site on their side inside the cutoff,
    so the default symmetric-site kernels evaluate that site alone there.
    Variant 8192 evaluates both sites as in the rest of the shell: the two
    flag the same border poses and agree within the FP32 summation order
    (energy at float32 storage, gradient 1e-6 relative), and both sit within
    the bar of the plain FP64 adjoint."""
    for case in (synth.small_field(), synth.batch_frameworks(1)[0]):
        size = 12
        _, axes = regular_pose_grid(size, 64)
        axes = normalized_directors(axes)
        shape = (64, size, size, size)
        with VextSystem(case) as system:
            res = {}
            for variant in (0, 8192):
                out = torch.empty(shape, dtype=torch.float32, device="cuda")
                grad = torch.empty(shape + (6,), dtype=torch.float32, device="cuda")
                batch = VextBatch([system], size, axes, [out], gradients=[grad],
                                  variant=variant)
                name = batch.info()["cta_shape"]
                assert ("two-site outer" in name) == (variant == 8192)
                batch.run()
                batch.check()
                res[variant] = (batch.refined(), out.cpu().numpy().astype(np.float64),
                                grad.cpu().numpy().astype(np.float64))
                batch.close()
            e64 = torch.empty(shape, dtype=torch.float64, device="cuda")
            g64 = torch.empty(shape + (6,), dtype=torch.float64, device="cuda")
            system.field_adjoint_device(size, axes, None, None, e64, g64,
                                        mode=_lib.VEXT_MODE_FP64_PLAIN)
            torch.cuda.synchronize()
        ex, gx = e64.cpu().numpy(), g64.cpu().numpy()
        (n1, e1, g1), (n2, e2, g2) = res[0], res[8192]
        assert n1 == n2
        assert (np.abs(e1 - e2) <= 2e-4 + 2.4e-7 * np.abs(e2)).all()
        rel = np.linalg.norm(g1 - g2, axis=-1) / np.maximum(np.linalg.norm(g2, axis=-1), 1.0)
        assert rel.max() < 1e-6
        for e, g in ((e1, g1), (e2, g2)):
            assert (np.abs(e - ex) <= 1e-4 + 1.2e-7 * np.abs(ex)).all()
            grel = np.linalg.norm(g - gx, axis=-1) / np.maximum(np.linalg.norm(gx, axis=-1), 1.0)
            assert grel.max() < 1e-5
