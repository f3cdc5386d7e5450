"""CPU restatement of one reference String iteration -- TEST INFRASTRUCTURE ONLY.

Only tests/ import this module, as the checker of the GPU String update.
It restates, in numpy, the kernels the reference solver runs per iteration
(native/string/source_code/RC_main.cu:1914-2390):

  s0_grad_cal, s0_grad_length_sqrt_cal   global.h:1281-1340  (gradient, truncation)
  s0_new_cal                             global.h:1347-1450  (normalised step)
  s1_fix_modify_upgrade                  global.h:1452-1620  (end fixing)
  s1_frac2cart, s1_length_prep, cumulation, s1_2_s2
                                         global.h:1622-1790  (reparametrisation)
  check_s2, smooth_angle                 global.h:1792-1905
  diff_s_prep, check_signal, copy2s0     global.h:2105-2244, legacy_policy.h:9-12

The gradient is pluggable: ``fd`` is the reference's own one-sided difference
(the oracle's restatement of Vext_s0_deri_cal), ``analytic`` is h x the FP64
oracle gradient (what the GPU update uses).  End fixing reads the values from
before fixing (the reference kernel runs all images at once).
"""
from __future__ import annotations

import numpy as np

from . import oracle

PI = 3.141592653589793


def _trunc(x, r):
    return np.floor(x / r) * r


def euler_director(s):
    b, g = s[:, 4], s[:, 5]
    return np.stack([np.cos(g) * np.cos(b), np.sin(g) * np.cos(b), -np.sin(b)], 1)


def analytic_gradient(case, s, hf, ha):
    """h_k dE/dx_k in (a, b, c, alpha, beta, gamma); dE/dalpha = 0."""
    cell = case["cell"]
    e, gc, gu = oracle.pose_energy_grad(case, s[:, :3] @ cell, euler_director(s))
    b, g = s[:, 4], s[:, 5]
    du_db = np.stack([-np.cos(g) * np.sin(b), -np.sin(g) * np.sin(b), -np.cos(b)], 1)
    du_dg = np.stack([-np.sin(g) * np.cos(b), np.cos(g) * np.cos(b), np.zeros_like(b)], 1)
    grad = np.column_stack([hf * (gc @ cell.T), np.zeros(len(s)), ha * (gu * du_db).sum(1),
                            ha * (gu * du_dg).sum(1)])
    return e, grad


def pose_energy(case, s):
    return oracle.pose_energy_grad(case, s[:, :3] @ case["cell"], euler_director(s))[0]


def smooth_one(prev, cur, nxt, k):
    dp, dn = prev - cur, nxt - cur
    if dp > PI:
        wrap = -2 * 2 * PI if dn > PI else -1 * 2 * PI
    elif dp < -PI:
        wrap = 2 * 2 * PI if dn < -PI else 0.0
    elif dn > PI:
        wrap = -1 * 2 * PI
    elif dn < -PI:
        wrap = 1 * 2 * PI
    else:
        wrap = 0.0
    return (1 - k) * cur + 0.5 * k * (prev + nxt + wrap)


def iteration(case, s0, hf=1e-4, ha=PI / 180, direction=1, smooth=1e-4, rounding=1e-15,
              conv_percent=30.0, check=False, gradient="analytic"):
    """One reference iteration.  Returns (new s0, stop flag, totals, e0)."""
    s0 = np.asarray(s0, dtype=float)
    n = len(s0)
    cell = case["cell"]
    if gradient == "fd":
        g = oracle.string_fd_gradient(case, s0, delta_frac=hf, delta_angle_rad=ha,
                                      rounding=rounding)
        e0 = pose_energy(case, s0)
    else:
        e0, g = analytic_gradient(case, s0, hf, ha)
        g = _trunc(g, rounding)
    lt = _trunc(np.sqrt((g[:, :3] ** 2).sum(1)), rounding)
    lr = _trunc(np.sqrt((g[:, 3:] ** 2).sum(1)), rounding)
    s1 = s0.copy()
    for i in range(n):
        for k in range(3):
            s1[i, k] = (s0[i, k] - hf * g[i, k] if lt[i] < hf
                        else s0[i, k] - hf * _trunc(g[i, k] / lt[i], rounding))
        for k in range(3, 6):
            s1[i, k] = (s0[i, k] - ha * g[i, k] if lr[i] < ha
                        else s0[i, k] - ha * _trunc(g[i, k] / lr[i], rounding))
    # end fixing (values from before fixing)
    d = direction - 1
    pre = s1.copy()
    s1[0, d] = s0[0, d]
    s1[n - 1, d] = s0[n - 1, d]
    for k in range(6):
        if k != d:
            s1[n - 1, k] = pre[0, k]
    for i in range(1, n - 1):
        v = pre[i, d]
        src = None
        if v < 0:
            src = next((ii for ii in range(i + 1, n) if pre[ii, d] > 0), None)
        elif v > 1:
            src = next((ii for ii in range(i - 1, -1, -1) if pre[ii, d] < 1), None)
        if src is not None:
            s1[i] = pre[src]
    # equal arc length in Cartesian space
    cart = s1[:, :3] @ cell
    seg = np.r_[0.0, np.sqrt(((cart[1:] - cart[:-1]) ** 2).sum(1))]
    cum = np.cumsum(seg)
    total = cum[-1]
    s2 = s1.copy()
    for i in range(n):
        t = i / (n - 1)
        ii = max(k for k in range(n - 1) if cum[k] / total <= t)
        l0, l1 = cum[ii] / total, cum[ii + 1] / total
        for k in range(3):
            s2[i, k] = (s1[ii, k] + (t - l0) * ((s1[ii + 1, k] - s1[ii, k]) / (l1 - l0))
                        if l1 > l0 else s1[ii, k])
    e2 = pose_energy(case, s2)
    for i in range(n):
        if e2[i] > e0[i]:
            s2[i, 3:] = s0[i, 3:]
    mt = np.sqrt(((s0[:, :3] - s2[:, :3]) ** 2).sum(1)).sum()
    mr = np.sqrt(((s0[:, 3:] - s2[:, 3:]) ** 2).sum(1)).sum()
    conv_t = conv_percent / 100 * hf * n * np.sqrt(3)
    conv_r = conv_percent / 100 * ha * n * np.sqrt(3)
    ct = np.isfinite(mt) and mt >= 0 and mt < conv_t
    cr = np.isfinite(mr) and mr >= 0 and mr < conv_r
    if check and ct and cr:
        return s0.copy(), True, (mt, mr), e0
    new = s2.copy()
    for i in range(1, n - 1):
        for k in range(3, 6):
            new[i, k] = smooth_one(s2[i - 1, k], s2[i, k], s2[i + 1, k], smooth)
    for k in range(3, 6):
        col = new[:, k]
        col = np.where(col > 2 * PI, col - 2 * PI, np.where(col < 0, col + 2 * PI, col))
        new[:, k] = col
    return new, False, (mt, mr), e0


def tst_diffusivity(frac, energy, cell, hop_A, temperature, mass_g_mol):
    """The String program's hopping diffusivity (RC_main.cu:2485-2527) restated:
    Cartesian arc length in m, trapezoid of exp(-V/T) capped at exp(-600),
    D0 = 0.5 L^2 sqrt(kT / (2 pi m)) exp(-Vmax / T) / trapz."""
    import math
    frac = np.asarray(frac, dtype=float)
    cell = np.asarray(cell, dtype=float)
    A, B, C = cell[:, 0], cell[:, 1], cell[:, 2]
    T = temperature
    xs = [(f[0] * A[0] + f[1] * A[1] + f[2] * A[2]) * 1e-10 for f in frac]
    ys = [(f[0] * B[0] + f[1] * B[1] + f[2] * B[2]) * 1e-10 for f in frac]
    zs = [(f[0] * C[0] + f[1] * C[1] + f[2] * C[2]) * 1e-10 for f in frac]
    s = [0.0]
    for i in range(1, len(frac)):
        s.append(s[-1] + math.sqrt((xs[i] - xs[i - 1]) ** 2 + (ys[i] - ys[i - 1]) ** 2
                                   + (zs[i] - zs[i - 1]) ** 2))
    w = [math.exp(-6e2) if e / T > 6e2 else math.exp(-e / T) for e in energy]
    integral = 0.0
    for i in range(1, len(frac)):
        integral = integral + (s[i] - s[i - 1]) * (w[i] + w[i - 1]) / 2
    vmax = energy[0]
    for e in energy:
        if e > vmax:
            vmax = e
    return (0.5 * (hop_A * 1e-10) ** 2
            * math.sqrt((1.38e-23 * T) / (2 * PI * (mass_g_mol / 1e3 / 6.02214076e23)))
            * (math.exp(-vmax / T) / integral))
