"""Regenerate the golden fixtures in this folder from the reference itself.

Run in a container where the reference project is importable (its Python
package under ``<reference>/src`` and its kernel compiled from source by
``make -C oracle ref``):

    python tests/golden/make_golden.py --reference /path/to/String_Vext

Every array stored here is an output of the reference's own code:
``direct_pose_energy`` and ``calculate_vext`` (src/string_vext/physics.py,
vext.py), its native kernel (native/vext/kernel.cpp built from source) driven
by its own ``NativeReusePotential`` (native.py), and its String pair function
(native/string/source_code/triclinic_pair.h, compiled through the reference's
host test shim).  Inputs are the seeded synthetic workloads of
``string_vext_b200.synth`` and the known-answer cases of the reference's
tests (tests/unit/test_public_api.py, test_native_string_triclinic.py).
"""
from __future__ import annotations

import argparse
import ctypes
import itertools
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]

#: The reference's own example input (a skewed cell, beta = 115.152 deg, one atom),
#: read from the reference checkout at generation time.
TOY_INPUT = Path("examples") / "toy_triclinic" / "input.dat"


def case_arrays(prefix, case):
    return {f"{prefix}_cell": case["cell"], f"{prefix}_frac": case["frame_frac"],
            f"{prefix}_sigma": case["frame_sigma"], f"{prefix}_epsilon": case["frame_epsilon"],
            f"{prefix}_guest": np.array([case["guest_epsilon"][0], case["guest_sigma"][0],
                                         case["bond_length"]]),
            f"{prefix}_cutoff": np.array(case["cutoff"])}


def main():
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--reference", type=Path, default=os.environ.get("VEXT_REFERENCE"),
                        help="reference checkout (default: $VEXT_REFERENCE)")
    args = parser.parse_args()
    if args.reference is None:
        parser.error("--reference (or $VEXT_REFERENCE) is required")
    args.reference = Path(args.reference)
    sys.path.insert(0, str(args.reference / "src"))
    sys.path.insert(0, str(REPO))
    from string_vext.input import parse_string_input
    from string_vext.native import NativeReusePotential
    from string_vext.orientation import regular_pose_grid
    from string_vext.physics import direct_pose_energy
    from string_vext.vext import calculate_vext

    from string_vext_b200 import synth

    kernel = REPO / "oracle/_ref/vext_kernel.so"
    pair_so = REPO / "oracle/_ref/pair.so"
    if not kernel.exists() or not pair_so.exists():
        raise SystemExit("build the reference objects first: make -C oracle ref")

    # 1. the reference unit test's toy skew cell (tests/unit/test_public_api.py:13-62)
    toy_text = (args.reference / TOY_INPUT).read_text()
    toy = parse_string_input(args.reference / TOY_INPUT)
    fields = calculate_vext(toy, size=3, orientations=4, kernel=kernel)
    c3, a4 = regular_pose_grid(3, 4)
    out = {"toy_input": np.array(toy_text), "toy_direct": direct_pose_energy(toy, c3, a4)}
    for key in ("orientation_K", "marginal_K", "site_K", "grid", "axes"):
        out[f"toy_{key}"] = fields[key]
    np.savez_compressed(HERE / "toy_skew.npz", **out)

    # 2. small_field at 4^3 x 64: direct, native and the full calculate_vext output
    case = synth.small_field()
    c4, a64 = regular_pose_grid(4, 64)
    direct = direct_pose_energy(case, c4, a64)
    native = NativeReusePotential(case, kernel).evaluate(c4, a64)
    fields = calculate_vext(case, size=4, orientations=64, kernel=kernel)
    out = {"direct": direct, "native": native, "centers": c4, "axes": a64}
    for key in ("orientation_K", "marginal_K", "site_K", "grid"):
        out[key] = fields[key]
    out.update(case_arrays("case", case))
    np.savez_compressed(HERE / "small_field_s4.npz", **out)

    # 3. sampled centers of the full-size and skewed workloads (all 64 directors)
    rng = np.random.default_rng(123)
    for name, maker in (("full_field", synth.full_field), ("skewed_field", synth.skewed_field)):
        case = maker()
        centers = np.vstack([rng.random((6, 3)), [[.001, .999, .5], [.999, .001, .02]]])
        direct = direct_pose_energy(case, centers, a64)
        native = NativeReusePotential(case, kernel).evaluate(centers, a64)
        np.savez_compressed(HERE / f"{name}_sample.npz", centers=centers, axes=a64,
                            direct=direct, native=native)

    # 4. the drop-in CSR kernel on one 512-center batch of small_field (bit-exact target)
    case = synth.small_field()
    c8, _ = regular_pose_grid(8, 64)
    pot = NativeReusePotential(case, kernel)
    cart = np.mod(c8, 1) @ pot.potential.cell
    groups = pot.potential.tree.query_ball_point(cart, pot.radius, workers=1)
    starts = np.zeros(len(groups) + 1, dtype=np.int64)
    starts[1:] = np.cumsum([len(g) for g in groups])
    indices = np.concatenate([np.asarray(g, dtype=np.int32) for g in groups])
    axes = a64 / np.linalg.norm(a64, axis=1, keepdims=True)
    lib = ctypes.CDLL(str(kernel))
    fn = lib.evaluate_reused_neighbors
    fn.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] + [ctypes.c_void_p] * 11
    fn.restype = ctypes.c_int
    output = np.zeros((len(cart), 64))
    arrays = [np.ascontiguousarray(x) for x in (cart, axes, pot.potential.images, pot.offsets,
                                                pot.coeff12, pot.coeff6, pot.shift, pot.floor2)]
    code = fn(len(cart), 64, len(arrays[2]), pot.cutoff**2,
              *(a.ctypes.data_as(ctypes.c_void_p) for a in arrays),
              starts.ctypes.data_as(ctypes.c_void_p), indices.ctypes.data_as(ctypes.c_void_p),
              output.ctypes.data_as(ctypes.c_void_p))
    assert code == 0
    np.savez_compressed(HERE / "csr_batch.npz", centers=arrays[0], axes=arrays[1],
                        offsets=arrays[3], cutoff2=np.array(pot.cutoff**2), starts=starts,
                        indices=indices, output=output, n_images=np.array(len(arrays[2])))

    # 5. String pair function known answers (test_native_string_triclinic.py:45-90)
    plib = ctypes.CDLL(str(pair_so))
    plib.run_triclinic_pair.argtypes = [ctypes.POINTER(ctypes.c_double)]
    plib.run_triclinic_pair.restype = ctypes.c_double

    def pair(cell, site, atom, sigma=3.5, epsilon=98., cutoff=5.5):
        p = np.r_[site, atom, cell.T.reshape(-1), epsilon, sigma, 50., 3.4, cutoff].astype(np.float64)
        return plib.run_triclinic_pair(p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    rows = []
    h = np.array([[10., 0., 0.], [8., 6., 0.], [0., 0., 10.]])
    rows.append((h, np.array([0., 0., 5.]), np.array([0., .9, .5]), 4.0))
    prng = np.random.default_rng(20260929)
    for h in (np.diag([9., 10., 11.]), np.array([[10., 0, 0], [4., 8., 0], [-3., 2., 9.]])):
        for _ in range(32):
            f, atom = prng.random((2, 3))
            rows.append((h, f @ h, atom, 5.5))
    rows.append((np.diag([4., 4., 4.]), np.array([2., 2., 2.]), np.array([.2, .3, .4]), 6.0))
    hp = np.array([[10., 0, 0], [4., 8., 0], [-3., 2., 9.]])
    fp, ap = np.array([.25, .35, .6]), np.array([.8, .1, .2])
    for shift in (np.zeros(3), np.array([3, -2, 1]), np.array([-5, 1, -4])):
        rows.append((hp, (fp + shift) @ hp, ap, 5.5))
        rows.append((hp, fp @ hp, ap + shift, 5.5))
    hc = np.diag([20., 20., 20.])
    rows.append((hc, np.array([.5, .5, .5]) @ hc, np.array([.5, .5, .5]), 5.5))
    rows.append((hc, np.array([.5, .5, .5]) @ hc + [5.5, 0, 0], np.array([.5, .5, .5]), 5.5))
    cells = np.array([r[0] for r in rows]); sites = np.array([r[1] for r in rows])
    atoms = np.array([r[2] for r in rows]); cutoffs = np.array([r[3] for r in rows])
    energy = np.array([pair(*r[:3], cutoff=r[3]) for r in rows])

    # brute force of the reference test (independent enumeration over [-5, 5]^3)
    def brute(cell, site, atom, sigma=3.5, epsilon=98., cutoff=5.5):
        shift = np.array(list(itertools.product(range(-5, 6), repeat=3)))
        guest = ((site @ np.linalg.inv(cell)) % 1) @ cell
        images = ((atom % 1)[None] + shift) @ cell
        r = np.linalg.norm(guest - images, axis=1)
        s = (sigma + 3.4) / 2; e = np.sqrt(epsilon * 50.)
        ratio = (s / np.maximum(r, .1 * s))**6; cut = (s / cutoff)**6
        return np.where(np.maximum(r, .1 * s) < cutoff, 4 * e * (ratio**2 - ratio - cut**2 + cut), 0.).sum()

    brute_e = np.array([brute(*r[:3], cutoff=r[3]) for r in rows])
    np.savez_compressed(HERE / "pair_lj.npz", cells=cells, sites=sites, atoms=atoms,
                        cutoffs=cutoffs, energy=energy, brute=brute_e)

    # 6. String pose energies (Euler convention) of small_field composed from the
    #    reference pair function: E = sum over sites and atoms of triclinic_pair_lj.
    case = synth.small_field()
    erng = np.random.default_rng(77)
    poses = np.column_stack([erng.random((6, 3)), erng.uniform(-np.pi, np.pi, (6, 3))])
    cell = case["cell"]

    def rot(a, b, g, v):
        ca, sa, cb, sb, cg, sg = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(g), np.sin(g)
        return np.array([v[0]*cg*cb - v[1]*sg*ca + v[1]*sa*cg*sb + v[2]*sg*sa + v[2]*ca*cg*sb,
                         v[0]*sg*cb + v[1]*cg*ca + v[1]*sg*sb*sa - v[2]*cg*sa + v[2]*sg*sb*ca,
                         -v[0]*sb + v[1]*cb*sa + v[2]*ca*cb])

    def pose_pair_energy(x):
        com = x[:3] @ cell
        total = 0.0
        for s in range(2):
            site = com + rot(x[3], x[4], x[5], case["guest_xyz"][s])
            for t in range(len(case["frame_frac"])):
                p = np.r_[site, case["frame_frac"][t], cell.T.reshape(-1),
                          case["guest_epsilon"][s], case["guest_sigma"][s],
                          case["frame_epsilon"][t], case["frame_sigma"][t],
                          case["cutoff"]].astype(np.float64)
                total += plib.run_triclinic_pair(p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return total

    e_poses = np.array([pose_pair_energy(x) for x in poses])
    np.savez_compressed(HERE / "euler_poses.npz", poses=poses, energy=e_poses)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
