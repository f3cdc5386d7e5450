// Pair loops shared by the per-field kernels (field.cu) and the persistent
// batched kernel (batch.cu): the staging protocol of one region's list and
// the per-chunk FP64 (near) and packed FP32x2 (far) pair sums.
//
// Pair term (native/vext/kernel.cpp:26-36 and neighbor.py:21-28):
//   d2 < rc^2:  s2 = max(d2, floor2), i6 = 1/s2^3, e = c12 i6^2 - c6 i6 + shift.
#pragma once

#include "stage.cuh"

namespace vext {

__device__ __forceinline__ float set_lt(float a, float b) {
    float r;
    asm("set.lt.f32.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// FP64 reciprocal: hardware seed (relative error <= 2^-23) refined by
// Newton-Raphson steps r' = r + r (1 - s r), each squaring the relative error
// and leaving it one-sided (r under-estimates): one step leaves <= 2^-46
// (1.4e-14, far below the mixed-precision bar), two reach FP64 rounding.
template <int STEPS = 2>
__device__ __forceinline__ double rcp64_nr(double s) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(s));
#pragma unroll
    for (int k = 0; k < STEPS; ++k) r = fma(r, fma(-s, r, 1.0), r);
    return r;
}

// ------------------------------------------------------------ staging

template <int NT>
__device__ __forceinline__ void load_types(float4 *stf, double *std4, const float4 *tf,
                                           const double *td, int n_types) {
    for (int t = threadIdx.x; t < n_types; t += NT) {
        stf[t] = tf[t];
        if (std4)
#pragma unroll
            for (int k = 0; k < 4; ++k) std4[4 * t + k] = td[4 * t + k];
    }
}

__device__ __forceinline__ void init_barriers(Stager &st) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&st.bar[s], 1);
        fence_mbar_init();
    }
}

// Chunk c of `plan` is the seq0 + c-th chunk this CTA stages: stage
// (seq0 + c) % kStages, phase parity ((seq0 + c) / kStages) & 1.
__device__ __forceinline__ void stage_prologue(Stager &st, const ChunkPlan &plan,
                                               const float4 *hi, const float4 *lo,
                                               unsigned seq0) {
    if (threadIdx.x == 0)
        for (int c = 0; c < min(kStages, plan.n_chunks); ++c) st.issue(plan, hi, lo, c, seq0 + c);
}

// Wait for chunk c; on a failed wait drain the copies in flight and report
// false (the whole CTA must then return).
__device__ __forceinline__ bool stage_wait(Stager &st, const ChunkPlan &plan, int c,
                                           unsigned seq0, int *status) {
    const unsigned q = seq0 + c;
    const bool ok = mbar_wait_bounded(&st.bar[q % kStages], (q / kStages) & 1, status);
    if (__syncthreads_and(ok)) return true;
    if (threadIdx.x == 0)
        for (int cc = c; cc < min(c + kStages, plan.n_chunks); ++cc)
            mbar_drain(&st.bar[(seq0 + cc) % kStages], ((seq0 + cc) / kStages) & 1);
    return false;
}

// All threads are done with chunk c: reuse its stage for chunk c + kStages.
__device__ __forceinline__ void stage_next(Stager &st, const ChunkPlan &plan, const float4 *hi,
                                           const float4 *lo, int c, unsigned seq0) {
    __syncthreads();
    if (threadIdx.x == 0 && c + kStages < plan.n_chunks)
        st.issue(plan, hi, lo, c + kStages, seq0 + c + kStages);
}

// Staged near chunk (hi + lo) -> FP64 (x, y, z, type) in shared memory.
template <int NT>
__device__ __forceinline__ void near_convert(const float4 *hb, const float4 *lb, double *ed,
                                             int len) {
    for (int e = threadIdx.x; e < len; e += NT) {
        const float4 h = hb[e], l = lb[e];
        ed[4 * e + 0] = (double)h.x + (double)l.x;
        ed[4 * e + 1] = (double)h.y + (double)l.y;
        ed[4 * e + 2] = (double)h.z + (double)l.z;
        ed[4 * e + 3] = (double)__float_as_int(h.w);
    }
}

// ------------------------------------------------------------ near (FP64)

struct NearGeom {
    double cx, cy, cz;        // grid center relative to the region origin
    double off0, off1;        // site offsets
    double m0, m1, oo0, oo1;  // -2 o_s and o_s^2
    double rc2;
    double floor_out2;        // |d0|^2 above which no site is inside a contact floor
};

__device__ __forceinline__ NearGeom near_geom(double cx, double cy, double cz, double off0,
                                              double off1, double rc2,
                                              double floor_out2 = 1e300) {
    NearGeom g;
    g.cx = cx;
    g.cy = cy;
    g.cz = cz;
    g.off0 = off0;
    g.off1 = off1;
    g.m0 = -2.0 * off0;
    g.m1 = -2.0 * off1;
    g.oo0 = off0 * off0;
    g.oo1 = off1 * off1;
    g.rc2 = rc2;
    g.floor_out2 = floor_out2;
    return g;
}

// Sum one converted near chunk into acc[p][site] for the thread's P directors.
//   MODE 0 (FP64 oracle): direct d = site - x per site, IEEE reciprocal,
//          cutoff test.
//   MODE 1/2 (mixed): the thread's poses share one grid center c, so with
//          d0 = x - c, t = d0 . u:  q_s = |d0|^2 + o_s^2 - 2 o_s t (|d0|^2
//          once per entry, 1 FMA per site after t); reciprocal refined
//          by one Newton step.  MODE 2 drops the cutoff test (near pairs are never
//          farther apart than r_split + 2 rho_site < rc, checked on the host)
//          and sums the shift once per entry into shift_sum (the caller adds
//          2 x shift_sum, both sites, to every energy); entries farther from
//          the center than NearGeom::floor_out2 skip the contact-floor test.
template <int P, int MODE>
__device__ __forceinline__ void near_chunk(const double *ed, const double *std4, int len,
                                           const NearGeom &g, const double (&ux)[P],
                                           const double (&uy)[P], const double (&uz)[P],
                                           double (&acc)[P][2], double &shift_sum) {
    const double2 *ed2 = reinterpret_cast<const double2 *>(ed);
    const double2 *td2 = reinterpret_cast<const double2 *>(std4);
#pragma unroll 1
    for (int e = 0; e < len; ++e) {
        const double2 xy = ed2[2 * e], zt = ed2[2 * e + 1];
        const int t = (int)zt.y;
        const double2 cc = td2[2 * t], sh = td2[2 * t + 1];   // (c12, c6), (shift, floor2)
        if (MODE == 0) {
#pragma unroll
            for (int p = 0; p < P; ++p)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const double off = q ? g.off1 : g.off0;
                    const double dx = g.cx + off * ux[p] - xy.x, dy = g.cy + off * uy[p] - xy.y,
                                 dz = g.cz + off * uz[p] - zt.x;
                    const double d2 = fma(dx, dx, fma(dy, dy, dz * dz));
                    const double s2 = fmax(d2, sh.y);
                    const double i2 = __drcp_rn(s2);
                    const double i6 = i2 * i2 * i2;
                    const double en = fma(i6, fma(cc.x, i6, -cc.y), sh.x);
                    acc[p][q] += d2 < g.rc2 ? en : 0.0;
                }
        } else {
            const double dx = xy.x - g.cx, dy = xy.y - g.cy, dz = zt.x - g.cz;
            const double dd = fma(dx, dx, fma(dy, dy, dz * dz));
            const double k0 = dd + g.oo0, k1 = dd + g.oo1;
            if (MODE == 2 && dd > g.floor_out2) {   // inside the cutoff, clear of every floor
                shift_sum += sh.x;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const double tt = fma(dx, ux[p], fma(dy, uy[p], dz * uz[p]));
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const double i2 = rcp64_nr<1>(fma(q ? g.m1 : g.m0, tt, q ? k1 : k0));
                        const double i6 = i2 * i2 * i2;
                        acc[p][q] = fma(i6, fma(cc.x, i6, -cc.y), acc[p][q]);
                    }
                }
                continue;
            }
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const double tt = fma(dx, ux[p], fma(dy, uy[p], dz * uz[p]));
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const double d2 = fma(q ? g.m1 : g.m0, tt, q ? k1 : k0);
                    const double s2 = fmax(d2, sh.y);
                    const double i2 = rcp64_nr<1>(s2);
                    const double i6 = i2 * i2 * i2;
                    const double en = fma(i6, fma(cc.x, i6, -cc.y), sh.x);
                    if (MODE == 1) acc[p][q] += d2 < g.rc2 ? en : 0.0;
                    else acc[p][q] += en;
                }
            }
        }
    }
}

// ------------------------------------------------------------ FP64 pose

// FP64 energy and site-force sums of one pose over entries k = first,
// first + step, ... of a region list (positions hi + lo relative to the
// region origin; c the grid center there, u the director):
//   e += sum over sites and in-cutoff pairs of c12 i6^2 - c6 i6 + shift,
//   g[0..2] += dE/dc, g[3..5] += dE/du (not yet projected),
// with d2 >= rc^2 out (the reference's test, kernel.cpp:29-30), the contact
// floor on d2 and no force below it.  It serves the plain FP64 kernels (one
// thread per pose); the FP64 re-evaluation of flagged poses (a warp per pose)
// uses fp64_pose_pairs_both, the same pair test and terms.
__device__ __forceinline__ void fp64_pose_pairs(const float4 *hi, const float4 *lo,
                                                const double *td, long long off, int n,
                                                int first, int step, double rc2, double off0,
                                                double off1, double cx, double cy, double cz,
                                                const double (&u)[3], double &e,
                                                double (&g)[6]) {
    for (int k = 0; k < 6; ++k) g[k] = 0.0;
    for (int s = 0; s < 2; ++s) {
        const double o = s ? off1 : off0;
        const double px = cx + o * u[0], py = cy + o * u[1], pz = cz + o * u[2];
        double gs[3] = {0, 0, 0};
        for (int k = first; k < n; k += step) {
            const float4 h = hi[off + k], l = lo[off + k];
            const double dx = px - ((double)h.x + (double)l.x);
            const double dy = py - ((double)h.y + (double)l.y);
            const double dz = pz - ((double)h.z + (double)l.z);
            const double d2 = fma(dx, dx, fma(dy, dy, dz * dz));
            if (d2 >= rc2) continue;
            const int t = __float_as_int(h.w);
            const double c12 = td[4 * t], c6 = td[4 * t + 1], fl = td[4 * t + 3];
            const double s2 = d2 < fl ? fl : d2;
            const double i2 = 1.0 / s2;
            const double i6 = i2 * i2 * i2;
            e += c12 * i6 * i6 - c6 * i6 + td[4 * t + 2];
            if (d2 >= fl) {
                const double de = 2.0 * (-6.0 * c12 * i6 * i6 + 3.0 * c6 * i6) * i2;
                gs[0] += de * dx;
                gs[1] += de * dy;
                gs[2] += de * dz;
            }
        }
        for (int k = 0; k < 3; ++k) {
            g[k] += gs[k];
            g[3 + k] += o * gs[k];
        }
    }
}

// fp64_pose_pairs for the re-evaluation of flagged poses: the same pair
// test (d2 from the same hi + lo sums and fma order, d2 >= rc^2 out, the
// contact floor) and terms, both sites per entry (each entry read once), and
// the reciprocal of d2 from the hardware seed and two Newton steps instead of
// a division (within an ulp or two of it).
__device__ __forceinline__ void fp64_pose_pairs_both(const float4 *hi, const float4 *lo,
                                                     const double *td, long long off, int n,
                                                     int first, int step, double rc2,
                                                     double off0, double off1, double cx,
                                                     double cy, double cz, const double (&u)[3],
                                                     double &e, double (&g)[6]) {
    const double p0x = cx + off0 * u[0], p0y = cy + off0 * u[1], p0z = cz + off0 * u[2];
    const double p1x = cx + off1 * u[0], p1y = cy + off1 * u[1], p1z = cz + off1 * u[2];
    double gs[2][3] = {{0, 0, 0}, {0, 0, 0}};
    for (int k = first; k < n; k += step) {
        const float4 h = hi[off + k], l = lo[off + k];
        const double ax = (double)h.x + (double)l.x, ay = (double)h.y + (double)l.y,
                     az = (double)h.z + (double)l.z;
        const int t = __float_as_int(h.w);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const double dx = (s ? p1x : p0x) - ax, dy = (s ? p1y : p0y) - ay,
                         dz = (s ? p1z : p0z) - az;
            const double d2 = fma(dx, dx, fma(dy, dy, dz * dz));
            if (d2 >= rc2) continue;
            const double c12 = td[4 * t], c6 = td[4 * t + 1], fl = td[4 * t + 3];
            const double s2 = d2 < fl ? fl : d2;
            const double i2 = rcp64_nr<2>(s2);
            const double i6 = i2 * i2 * i2;
            e += c12 * i6 * i6 - c6 * i6 + td[4 * t + 2];
            if (d2 >= fl) {
                const double de = 2.0 * (-6.0 * c12 * i6 * i6 + 3.0 * c6 * i6) * i2;
                gs[s][0] += de * dx;
                gs[s][1] += de * dy;
                gs[s][2] += de * dz;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) g[k] = 0.0;
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            g[k] += gs[s][k];
            g[3 + k] += (s ? off1 : off0) * gs[s][k];
        }
}

// Project dE/du (g[3..5]) on the plane normal to the unit director u.
__device__ __forceinline__ void fp64_tangent(const double (&u)[3], double (&g)[6]) {
    const double uu = g[3] * u[0] + g[4] * u[1] + g[5] * u[2];
    for (int k = 0; k < 3; ++k) g[3 + k] -= uu * u[k];
}


// ------------------------------------------------------------ far (FP32x2)

struct FarGeom {
    float cx, cy, cz;          // grid center (FP32) relative to the region origin
    float2 m0, m1;             // -2 o_s, broadcast
    float oo0, oo1;            // o_s^2
    float rc2f;
    float out2;                // |d0|^2 beyond which no site of the pose reaches rc
    // symmetric sites (o_1 = -o_0 = -o): q_s = rc^2 where s (d0 . u) = T* =
    // (|d0|^2 + o^2 - rc^2) / (2 o) = |d0|^2 inv2o + tb
    float inv2o, tb;
};

__device__ __forceinline__ FarGeom far_geom(double cxd, double cyd, double czd, double off0,
                                            double off1, float rc2f) {
    FarGeom g;
    g.cx = (float)cxd;
    g.cy = (float)cyd;
    g.cz = (float)czd;
    g.m0 = make_float2(-2.f * (float)off0, -2.f * (float)off0);
    g.m1 = make_float2(-2.f * (float)off1, -2.f * (float)off1);
    g.oo0 = (float)(off0 * off0);
    g.oo1 = (float)(off1 * off1);
    g.rc2f = rc2f;
    // (rc + max|o| + 1e-3 A)^2: a site is at least |d0| - max|o| from the
    // entry, so beyond this every pair is out by far more than FP32 rounding
    const double rmax = sqrt((double)rc2f) + fmax(fabs(off0), fabs(off1)) + 1e-3;
    g.out2 = (float)(rmax * rmax);
    const double inv2o = off0 != 0.0 ? 1.0 / (2.0 * off0) : 0.0;
    g.inv2o = (float)inv2o;
    g.tb = (float)((off0 * off0 - (double)rc2f) * inv2o);
    return g;
}

// A shell pair is classified by the FP32 test (q < rc^2 in FP32) as by the
// FP64 one unless its FP32 q lies within kBorderTol (A^2) of rc^2.  Worst
// case, every error aligned, for |d0| <= 13.4 A: each d0 component off by
// <= 9.9e-7 A (entry and center rounded to FP32, then the subtraction),
// which moves |d0|^2 by <= 2 |d0| sqrt(3) 9.9e-7 = 4.6e-5; the roundings of
// |d0|^2 (3 x 7.6e-6), of t = d0 . u with FP32 u (moving q by <= 5e-6), of
// |d0|^2 + o^2 and of the site FMA (7.6e-6 each); rc^2 rounded to FP32
// (7.6e-6): <= 9.8e-5 in all.
constexpr float kBorderTol = 1.25e-4f;
// The per-director test estimates min_s |q_s - rc^2| as 2 |o| | |t| - |T*| |
// from the same FP32 |d0|^2 and t; T* (rounded 1/(2o), offset and FMA) and
// the missing site roundings put that estimate within 3.6e-5 of the FP32
// q's own distance, so the director test flags below kBorderTol + 4e-5.
constexpr float kBorderTolDir = kBorderTol + 4e-5f;

// One far (site, atom) pair in FP64 for a site whose FP32 d2 lies within
// kBorderTol of rc^2: the oracle's test (d2 >= rc^2 out) decides it; inside,
// its energy (with the shift) is added to e and its site force dE/dsite =
// 2 (dE/dd2) (site - x) to f.  Far pairs lie beyond every contact floor.
__device__ __forceinline__ void fp64_border_pair(double sx, double sy, double sz, double ax,
                                                 double ay, double az, const double *td, int ty,
                                                 double rc2, double &e, double *f) {
    const double dx = sx - ax, dy = sy - ay, dz = sz - az;
    const double d2 = fma(dx, dx, fma(dy, dy, dz * dz));
    if (d2 >= rc2) return;
    const double c12 = td[4 * ty], c6 = td[4 * ty + 1];
    const double i2 = rcp64_nr<2>(d2);
    const double i6 = i2 * i2 * i2;
    e += fma(i6, fma(c12, i6, -c6), td[4 * ty + 2]);
    const double w = i2 * i6 * fma(-12.0 * c12, i6, 6.0 * c6);
    f[0] = fma(w, dx, f[0]);
    f[1] = fma(w, dy, f[1]);
    f[2] = fma(w, dz, f[2]);
}

// Border repair of one pose (entries k = first, first + step, ... of the
// shell range [off, off + n) of its region list): for each site, the far
// kernel's FP32 inside/outside decision -- recomputed with exactly its
// operations (far_geom, far_chunk_adj: d0 = hi - c in FP32, |d0|^2 and
// d0 . u as fused multiply-adds in the same order, q = m t + (|d0|^2 + o^2),
// inside when q < rc^2 in FP32) -- against the FP64 one (hi + lo positions,
// d2 >= rc^2 out).  A pair inside in FP64 only adds its FP64 energy (with
// the shift) and gradient terms to e and g; inside in FP32 only subtracts
// them.  Entries the far kernel skipped (|d0|^2 beyond FarGeom::out2) are
// out in both, and so are pairs whose FP32 q lies kBorderTol or more from
// rc^2 (only the FP32 terms are formed for those).  Shell pairs lie far
// beyond every contact floor.
__device__ __forceinline__ void shell_border_repair(const float4 *hi, const float4 *lo,
                                                    const double *td, long long off, int n,
                                                    int first, int step, double rc2,
                                                    float rc2f, double off0, double off1,
                                                    double cx, double cy, double cz,
                                                    const double (&u)[3], double &e,
                                                    double (&g)[6]) {
    const FarGeom f = far_geom(cx, cy, cz, off0, off1, rc2f);
    const float ufx = (float)u[0], ufy = (float)u[1], ufz = (float)u[2];
    e = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) g[k] = 0.0;
    // four entries per lane and round, their loads issued together (the
    // per-entry work is short: one load at a time left the loop waiting on
    // memory); each lane still visits its entries in increasing order
    constexpr int kRound = 4;
#pragma unroll 1
    for (int k0 = first; k0 < n; k0 += kRound * step) {
        float4 hv[kRound];
#pragma unroll
        for (int i = 0; i < kRound; ++i) {
            const int k = k0 + i * step;
            hv[i] = k < n ? hi[off + k] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < kRound; ++i) {
        const int k = k0 + i * step;
        if (k >= n) continue;
        const float4 h = hv[i];
        const float dx = h.x - f.cx, dy = h.y - f.cy, dz = h.z - f.cz;
        const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (dd > f.out2) continue;
        const float t = fmaf(dx, ufx, fmaf(dy, ufy, dz * ufz));
        const float q0 = fmaf(f.m0.x, t, dd + f.oo0), q1 = fmaf(f.m1.x, t, dd + f.oo1);
        // beyond kBorderTol of rc^2 the FP32 decision is the FP64 one
        if (fabsf(q0 - rc2f) >= kBorderTol && fabsf(q1 - rc2f) >= kBorderTol) continue;
        const float4 l = lo[off + k];
        const double ax = (double)h.x + (double)l.x, ay = (double)h.y + (double)l.y,
                     az = (double)h.z + (double)l.z;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const float q32 = s ? q1 : q0;
            const double os = s ? off1 : off0;
            const double px = cx + os * u[0] - ax, py = cy + os * u[1] - ay,
                         pz = cz + os * u[2] - az;
            const double d2 = fma(px, px, fma(py, py, pz * pz));
            const bool in32 = q32 < rc2f, in64 = d2 < rc2;
            if (in32 == in64) continue;
            const int ty = __float_as_int(h.w);
            const double c12 = td[4 * ty], c6 = td[4 * ty + 1];
            const double i2 = rcp64_nr<2>(d2);
            const double i6 = i2 * i2 * i2;
            const double w = in64 ? 1.0 : -1.0;
            e += w * (c12 * i6 * i6 - c6 * i6 + td[4 * ty + 2]);
            const double de = w * 2.0 * (-6.0 * c12 * i6 * i6 + 3.0 * c6 * i6) * i2;
            g[0] += de * px;
            g[1] += de * py;
            g[2] += de * pz;
            g[3] += os * de * px;
            g[4] += os * de * py;
            g[5] += os * de * pz;
        }
        }
    }
}

// The earlier forward far chunk, kept for comparison with far_chunk_fwd:
// per lane n3 = hardware reciprocal of -q^3, refined (NEWTON) by n3' = n3 +
// n3 (1 + q^3 n3); e = n3 (c12 n3 + c6) + shift = c12/q^6 - c6/q^3 + shift;
// a 1/0 mask (q < rc^2) multiplies e into FP32 partial sums flushed into FP64
// every FLUSH entries.  Far entries are >= r_split from every site, so no
// pair reaches the contact floor (no max()).
template <int P, bool NEWTON, int FLUSH>
__device__ __forceinline__ void far_chunk(const float4 *hb, const float4 *stf, int len,
                                          const FarGeom &g, const float2 (&ux)[P / 2],
                                          const float2 (&uy)[P / 2], const float2 (&uz)[P / 2],
                                          double (&acc)[P]) {
    constexpr int PP = P / 2;
    const float2 one2 = make_float2(1.f, 1.f);
#pragma unroll 1
    for (int e0 = 0; e0 < len; e0 += FLUSH) {
        float2 fa[PP];
#pragma unroll
        for (int j = 0; j < PP; ++j) fa[j] = make_float2(0.f, 0.f);
        const int e1 = min(e0 + FLUSH, len);
#pragma unroll 2
        for (int e = e0; e < e1; ++e) {
            const float4 h = hb[e];
            const float4 tp = stf[__float_as_int(h.w)];   // (c12, c6, shift, floor2)
            const float dx = h.x - g.cx, dy = h.y - g.cy, dz = h.z - g.cz;
            const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float2 k0 = make_float2(dd + g.oo0, dd + g.oo0),
                         k1 = make_float2(dd + g.oo1, dd + g.oo1);
            const float2 dx2 = make_float2(dx, dx), dy2 = make_float2(dy, dy),
                         dz2 = make_float2(dz, dz);
            const float2 c12 = make_float2(tp.x, tp.x), c6 = make_float2(tp.y, tp.y),
                         sh = make_float2(tp.z, tp.z);
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                const float2 t =
                    __ffma2_rn(dx2, ux[j], __ffma2_rn(dy2, uy[j], __fmul2_rn(dz2, uz[j])));
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const float2 d2 = __ffma2_rn(q ? g.m1 : g.m0, t, q ? k1 : k0);
                    const float2 d6 = __fmul2_rn(__fmul2_rn(d2, d2), d2);
                    float r0, r1;
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(-d6.x));
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(-d6.y));
                    float2 n3 = make_float2(r0, r1);
                    if (NEWTON) n3 = __ffma2_rn(n3, __ffma2_rn(d6, n3, one2), n3);
                    const float2 en = __ffma2_rn(n3, __ffma2_rn(c12, n3, c6), sh);
                    const float2 m = make_float2(set_lt(d2.x, g.rc2f), set_lt(d2.y, g.rc2f));
                    fa[j] = __ffma2_rn(en, m, fa[j]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < PP; ++j) {
            acc[2 * j] += (double)fa[j].x;
            acc[2 * j + 1] += (double)fa[j].y;
        }
    }
}

// Forward far chunk, the default: per lane n1 = hardware reciprocal of q (no
// Newton step), n3 = n1^3 = q^-3, e = n3 (c12 n3 - c6); MASK as in
// far_chunk_adj (inner entries: no mask, shift summed once per entry into
// shift_sum, to be added twice -- both sites -- to every energy).  FP32
// partials over FLUSH entries are flushed into the FP64 acc.  Shell entries
// beyond every site's cutoff (the list radius carries the region radius on
// top) are skipped: they would add exactly nothing.
// OUTER (symmetric sites, MASK): entries [outer_from, len) are outer shell
// entries (RegionInfo::n_outer: |d0| > rc for every pose center of the
// region), where a director's site on the far side of the center has q >=
// |d0|^2 + o^2 > rc^2 and adds exact zeros; only the near site (q = |d0|^2 +
// o^2 - |2 o t|, the same FP32 fma as its two-site q) is evaluated there, so
// the partials, and the result, are bit for bit those of the two-site loop.
template <int P, int FLUSH, bool MASK, bool OUTER = false>
__device__ __forceinline__ void far_chunk_fwd(const float4 *hb, const float4 *stf, int len,
                                              const FarGeom &g, const float2 (&ux)[P / 2],
                                              const float2 (&uy)[P / 2],
                                              const float2 (&uz)[P / 2], double (&acc)[P],
                                              double &shift_sum, int outer_from = 0) {
    static_assert(!OUTER || MASK, "outer entries are shell entries");
    constexpr int PP = P / 2;
    const float2 nam = make_float2(-fabsf(g.m0.x), -fabsf(g.m0.x));   // -|m0|
#pragma unroll 1
    for (int e0 = 0; e0 < len; e0 += FLUSH) {
        float2 fa[PP];
        float fs = 0.f;
#pragma unroll
        for (int j = 0; j < PP; ++j) fa[j] = make_float2(0.f, 0.f);
        const int e1 = min(e0 + FLUSH, len);
        const int em = OUTER ? max(e0, min(e1, outer_from)) : e1;
#pragma unroll 2
        for (int e = e0; e < em; ++e) {
            float2 k0, k1, dx2, dy2, dz2, c12, mc6, sh;
            {
                const float4 h = hb[e];
                const float4 tp = stf[__float_as_int(h.w)];   // (c12, c6, shift, -)
                const float dx = h.x - g.cx, dy = h.y - g.cy, dz = h.z - g.cz;
                const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                if (MASK && dd > g.out2) continue;
                k0 = make_float2(dd + g.oo0, dd + g.oo0);
                k1 = make_float2(dd + g.oo1, dd + g.oo1);
                dx2 = make_float2(dx, dx);
                dy2 = make_float2(dy, dy);
                dz2 = make_float2(dz, dz);
                c12 = make_float2(tp.x, tp.x);
                mc6 = make_float2(-tp.y, -tp.y);
                sh = make_float2(tp.z, tp.z);
                if (!MASK) fs += tp.z;
            }
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                const float2 t =
                    __ffma2_rn(dx2, ux[j], __ffma2_rn(dy2, uy[j], __fmul2_rn(dz2, uz[j])));
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const float2 d2 = __ffma2_rn(q ? g.m1 : g.m0, t, q ? k1 : k0);
                    float r0, r1;
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(d2.x));
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(d2.y));
                    const float2 n1 = make_float2(r0, r1);
                    float2 n3 = __fmul2_rn(__fmul2_rn(n1, n1), n1);
                    if (MASK) {
                        const float2 m = make_float2(set_lt(d2.x, g.rc2f), set_lt(d2.y, g.rc2f));
                        n3 = __fmul2_rn(n3, m);
                        fa[j] = __ffma2_rn(m, sh, fa[j]);
                    }
                    fa[j] = __ffma2_rn(n3, __ffma2_rn(c12, n3, mc6), fa[j]);
                }
            }
        }
        if (OUTER) {
#pragma unroll 2
            for (int e = em; e < e1; ++e) {   // outer entries: the near site alone
                float2 k0, dx2, dy2, dz2, c12, mc6, sh;
                {
                    const float4 h = hb[e];
                    const float4 tp = stf[__float_as_int(h.w)];
                    const float dx = h.x - g.cx, dy = h.y - g.cy, dz = h.z - g.cz;
                    const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    if (dd > g.out2) continue;
                    k0 = make_float2(dd + g.oo0, dd + g.oo0);
                    dx2 = make_float2(dx, dx);
                    dy2 = make_float2(dy, dy);
                    dz2 = make_float2(dz, dz);
                    c12 = make_float2(tp.x, tp.x);
                    mc6 = make_float2(-tp.y, -tp.y);
                    sh = make_float2(tp.z, tp.z);
                }
#pragma unroll
                for (int j = 0; j < PP; ++j) {
                    const float2 t =
                        __ffma2_rn(dx2, ux[j], __ffma2_rn(dy2, uy[j], __fmul2_rn(dz2, uz[j])));
                    const float2 d2 = __ffma2_rn(nam, make_float2(fabsf(t.x), fabsf(t.y)), k0);
                    float r0, r1;
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(d2.x));
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(d2.y));
                    const float2 n1 = make_float2(r0, r1);
                    float2 n3 = __fmul2_rn(__fmul2_rn(n1, n1), n1);
                    const float2 m = make_float2(set_lt(d2.x, g.rc2f), set_lt(d2.y, g.rc2f));
                    n3 = __fmul2_rn(n3, m);
                    fa[j] = __ffma2_rn(m, sh, fa[j]);
                    fa[j] = __ffma2_rn(n3, __ffma2_rn(c12, n3, mc6), fa[j]);
                }
            }
        }
        if (!MASK) shift_sum += (double)fs;
#pragma unroll
        for (int j = 0; j < PP; ++j) {
            acc[2 * j] += (double)fa[j].x;
            acc[2 * j + 1] += (double)fa[j].y;
        }
    }
}

// ------------------------------------------------------------ adjoint
//
// Forward + adjoint sums of one pose (center c, unit director u, sites at
// c + o_s u).  With d0 = x - c and q_s = |d0 - o_s u|^2 = |d0|^2 + o_s^2 -
// 2 o_s (d0 . u), every pair contributes through fp_s = (dE/dq_s) / 3 =
// q^-4 (c6 - 2 c12 q^-3)  (zero beyond the cutoff and on the contact floor):
//   dE/dc = -6 (sum_s H_s - u sum_s o_s F_s)
//   dE/du = -6 (sum_s o_s H_s) + (terms along u, removed by the tangent
//           projection),
// with H_s = sum_x fp_s d0 and F_s = sum_x fp_s.  For symmetric sites (o_1 =
// -o_0) only F_0 - F_1 enters (sum_s o_s F_s = o_0 (F_0 - F_1)): the SYM
// loops keep it in f[0] and leave f[1] at zero.  AdjAcc holds E, H_s, F_s of
// one director in FP64.
struct AdjAcc {
    double e, h[2][3], f[2];
};

template <int P>
__device__ __forceinline__ void adj_zero(AdjAcc (&acc)[P]) {
#pragma unroll
    for (int p = 0; p < P; ++p) {
        acc[p].e = 0.0;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            acc[p].f[q] = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[p].h[q][k] = 0.0;
        }
    }
}

// Energy and the six gradient components (dE/dc, tangent dE/du) of one
// director from its sums.
__device__ __forceinline__ void adj_finish(const AdjAcc &a, double off0, double off1, double ux,
                                           double uy, double uz, double &e, double (&g)[6]) {
    const double u[3] = {ux, uy, uz};
    const double sw = off0 * a.f[0] + off1 * a.f[1];
    double w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        g[k] = -6.0 * (a.h[0][k] + a.h[1][k] - u[k] * sw);
        w[k] = -6.0 * (off0 * a.h[0][k] + off1 * a.h[1][k]);
    }
    const double wu = w[0] * u[0] + w[1] * u[1] + w[2] * u[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) g[3 + k] = w[k] - wu * u[k];
    e = a.e;
}

// The pairs of one near entry (d0 = entry - center, dd = |d0|^2) with the
// thread's P directors, forward + adjoint.  FLOOR: some site may lie inside
// the entry type's contact floor (d2 < floor2: energy at the floor, no
// force); without it the floor tests are left out (the caller checks dd
// against NearGeom::floor_out2 so that every site is clear of every floor).
template <int P, int MODE, bool FLOOR, bool SYM>
__device__ __forceinline__ void near_entry_adj(double dx, double dy, double dz, double dd,
                                               double2 cc, double2 sh, const NearGeom &g,
                                               const double (&ux)[P], const double (&uy)[P],
                                               const double (&uz)[P], AdjAcc (&acc)[P]) {
    const double m2c12 = -2.0 * cc.x;
    // SYM: o_1 = -o_0, so q_1 = k0 - m0 t
    const double k0 = dd + g.oo0, k1 = SYM ? k0 : dd + g.oo1;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const double tt = fma(dx, ux[p], fma(dy, uy[p], dz * uz[p]));
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const double d2 = fma(q ? (SYM ? -g.m0 : g.m1) : g.m0, tt, q ? k1 : k0);
            const double s2 = FLOOR ? fmax(d2, sh.y) : d2;
            const double i2 = rcp64_nr<1>(s2);
            const double i6 = i2 * i2 * i2;
            double fp = (i6 * i2) * fma(m2c12, i6, cc.y);
            if (FLOOR) fp = d2 < sh.y ? 0.0 : fp;
            if (MODE == 1) {
                const bool in = d2 < g.rc2;
                acc[p].e += in ? fma(i6, fma(cc.x, i6, -cc.y), sh.x) : 0.0;
                fp = in ? fp : 0.0;
            } else {
                acc[p].e = fma(i6, fma(cc.x, i6, -cc.y), acc[p].e);   // shift: per entry
            }
            acc[p].h[q][0] = fma(fp, dx, acc[p].h[q][0]);
            acc[p].h[q][1] = fma(fp, dy, acc[p].h[q][1]);
            acc[p].h[q][2] = fma(fp, dz, acc[p].h[q][2]);
            if (SYM) acc[p].f[0] += q ? -fp : fp;
            else acc[p].f[q] += fp;
        }
    }
}

// FP64 near chunk, forward + adjoint (MODE 1: cutoff test, MODE 2: none);
// same centre-based q as near_chunk.  MODE 2 (every pair inside the cutoff):
// the shift, the same for every pose, is summed once per entry into
// shift_sum (the caller adds 2 x shift_sum, both sites, to every energy).
// Entries farther than NearGeom::floor_out2 from the center take the pair
// loop without the contact-floor tests (nearly all of them; the branch is
// uniform across the warp but for entries right at that radius).
template <int P, int MODE, bool SYM = false>
__device__ __forceinline__ void near_chunk_adj(const double *ed, const double *std4, int len,
                                               const NearGeom &g, const double (&ux)[P],
                                               const double (&uy)[P], const double (&uz)[P],
                                               AdjAcc (&acc)[P], double &shift_sum) {
    static_assert(MODE == 1 || MODE == 2, "mixed modes only");
    const double2 *ed2 = reinterpret_cast<const double2 *>(ed);
    const double2 *td2 = reinterpret_cast<const double2 *>(std4);
#pragma unroll 1
    for (int e = 0; e < len; ++e) {
        const double2 xy = ed2[2 * e], zt = ed2[2 * e + 1];
        const int t = (int)zt.y;
        const double2 cc = td2[2 * t], sh = td2[2 * t + 1];   // (c12, c6), (shift, floor2)
        const double dx = xy.x - g.cx, dy = xy.y - g.cy, dz = zt.x - g.cz;
        const double dd = fma(dx, dx, fma(dy, dy, dz * dz));
        if (MODE == 2) shift_sum += sh.x;
        if (dd > g.floor_out2)
            near_entry_adj<P, MODE, false, SYM>(dx, dy, dz, dd, cc, sh, g, ux, uy, uz, acc);
        else
            near_entry_adj<P, MODE, true, SYM>(dx, dy, dz, dd, cc, sh, g, ux, uy, uz, acc);
    }
}

// Shared-memory home of the FP64 gradient sums (H_s, F_s) of a CTA for
// kernels that keep only the energy sums in registers during the far passes:
// component k (0-2 = h[0], 3-5 = h[1], 6-7 = f) of director p of thread t is
// gsum[(p * kGradWords + k) * NT + t] (consecutive threads, consecutive words).
constexpr int kGradWords = 8;

template <int NT>
__device__ __forceinline__ double &grad_slot(double *gsum, int p, int k) {
    return gsum[(p * kGradWords + k) * NT + threadIdx.x];
}

// Directors p0 .. p0 + P - 1 of the shared-memory sums from acc.
// (SYM: f[1] stays zero and is neither stored nor loaded.)
template <int NT, int P, bool SYM = false>
__device__ __forceinline__ void grad_store(double *gsum, const AdjAcc (&acc)[P], int p0 = 0) {
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
#pragma unroll
            for (int k = 0; k < 3; ++k)
                grad_slot<NT>(gsum, p0 + p, 3 * q + k) = acc[p].h[q][k];
            if (!SYM || q == 0) grad_slot<NT>(gsum, p0 + p, 6 + q) = acc[p].f[q];
        }
}

template <int NT, int P, bool SYM = false>
__device__ __forceinline__ void grad_load(double *gsum, AdjAcc (&acc)[P]) {
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[p].h[q][k] = grad_slot<NT>(gsum, p, 3 * q + k);
            if (!SYM || q == 0) acc[p].f[q] = grad_slot<NT>(gsum, p, 6 + q);
        }
}

// Packed FP32x2 far chunk, forward + adjoint (lanes = two directors).  Per
// site, by default (RCP1): n1 = hardware reciprocal of q per lane, n3 = n1^3 =
// q^-3, e = n3 (c12 n3 - c6) + m shift, fp = (n1 n3) (c6 - 2 c12 n3) =
// (dE/dq) / 3, with m the 1/0 cutoff mask folded into n3.  The alternative
// (RCP1 = false): n3 = reciprocal of -q^3, e = n3 (c12 n3 + c6), fp = n3 (2 c12
// n3 + c6) (n3 q^2).  NEWTON refines the reciprocal by one Newton step.
// MASK = false for inner entries (inside the cutoff of every site of every
// pose of the region): no mask, and the shift, the same for every pose, is
// summed once per entry into shift_sum (the caller adds 2 x shift_sum, both
// sites, to every energy).  FP32 partials are flushed into the FP64 AdjAcc:
// the energy every 16 entries, the gradient sums every FLUSH entries.
// GSUM_NT > 0: the gradient partials go to the shared-memory sums
// (grad_slot<GSUM_NT>(gsum, ...)) instead of acc (whose energies stay).
// border (masked entries only, when non-null): per director the smallest
// |q - rc^2| met, so that poses with a pair whose FP32 q lies too close to
// the cutoff for the FP32 test to decide it like the FP64 one can be
// re-evaluated in FP64 (the force jumps at rc, so a pair counted on the
// other side moves the gradient by the jump).
// Shell entries beyond every site's cutoff are skipped (they add exactly
// nothing).
template <int P, bool NEWTON, int FLUSH, bool MASK, bool RCP1 = true, int UNROLL = 1,
          int GSUM_NT = 0, int BORDER = 0, bool SYM = false>
__device__ __forceinline__ void far_chunk_adj(const float4 *hb, const float4 *stf, int len,
                                              const FarGeom &g, const float2 (&ux)[P / 2],
                                              const float2 (&uy)[P / 2],
                                              const float2 (&uz)[P / 2], AdjAcc (&acc)[P],
                                              double &shift_sum, double *gsum = nullptr,
                                              float *border = nullptr) {
    constexpr int PP = P / 2;
    const float2 one2 = make_float2(1.f, 1.f);
    const float2 mrc2 = make_float2(-g.rc2f, -g.rc2f);
#pragma unroll 1
    for (int e0 = 0; e0 < len; e0 += FLUSH) {
        float2 fh[PP][2][3], ff[PP][2];
#pragma unroll
        for (int j = 0; j < PP; ++j)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                ff[j][q] = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < 3; ++k) fh[j][q][k] = make_float2(0.f, 0.f);
            }
        const int e1 = min(e0 + FLUSH, len);
#pragma unroll 1
        for (int b0 = e0; b0 < e1; b0 += 16) {   // energy partials: 16 entries
        float2 fe[PP];
        float fs = 0.f;
#pragma unroll
        for (int j = 0; j < PP; ++j) fe[j] = make_float2(0.f, 0.f);
        const int b1 = min(b0 + 16, e1);
#pragma unroll UNROLL
        for (int e = b0; e < b1; ++e) {
            float2 k0, k1, dx2, dy2, dz2, c12, c6, sh, mc6, m2c12;
            float4 tp;
            float ts = 0.f;
            {
                const float4 h = hb[e];
                tp = stf[__float_as_int(h.w)];   // (c12, c6, shift, -)
                const float dx = h.x - g.cx, dy = h.y - g.cy, dz = h.z - g.cz;
                const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                if (MASK && dd > g.out2) continue;
                k0 = make_float2(dd + g.oo0, dd + g.oo0);
                if (!SYM) k1 = make_float2(dd + g.oo1, dd + g.oo1);   // SYM: o_1^2 = o_0^2
                dx2 = make_float2(dx, dx);
                dy2 = make_float2(dy, dy);
                dz2 = make_float2(dz, dz);
                c12 = make_float2(tp.x, tp.x);
                c6 = make_float2(tp.y, tp.y);
                sh = make_float2(tp.z, tp.z);
                mc6 = make_float2(-tp.y, -tp.y);
                m2c12 = make_float2(-2.f * tp.x, -2.f * tp.x);
                if (!MASK) fs += tp.z;
                if (BORDER == 2) ts = fabsf(fmaf(dd, g.inv2o, g.tb));
            }
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                const float2 t =
                    __ffma2_rn(dx2, ux[j], __ffma2_rn(dy2, uy[j], __fmul2_rn(dz2, uz[j])));
                if (MASK && BORDER == 2) {
                    border[2 * j] = fminf(border[2 * j], fabsf(fabsf(t.x) - ts));
                    border[2 * j + 1] = fminf(border[2 * j + 1], fabsf(fabsf(t.y) - ts));
                }
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const float2 d2 = __ffma2_rn(q ? g.m1 : g.m0, t, q && !SYM ? k1 : k0);
                    float2 fp;
                    if (RCP1) {
                        float r0, r1;
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(d2.x));
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(d2.y));
                        float2 n1 = make_float2(r0, r1);
                        if (NEWTON)
                            n1 = __ffma2_rn(n1, __ffma2_rn(make_float2(-d2.x, -d2.y), n1, one2),
                                            n1);
                        float2 n3 = __fmul2_rn(__fmul2_rn(n1, n1), n1);
                        if (MASK) {
                            const float2 m =
                                make_float2(set_lt(d2.x, g.rc2f), set_lt(d2.y, g.rc2f));
                            n3 = __fmul2_rn(n3, m);
                            fe[j] = __ffma2_rn(m, sh, fe[j]);
                            if (BORDER == 1) {
                                const float2 x = __fadd2_rn(d2, mrc2);
                                border[2 * j] = fminf(border[2 * j], fabsf(x.x));
                                border[2 * j + 1] = fminf(border[2 * j + 1], fabsf(x.y));
                            }
                        }
                        fe[j] = __ffma2_rn(n3, __ffma2_rn(c12, n3, mc6), fe[j]);
                        fp = __fmul2_rn(__fmul2_rn(n1, n3), __ffma2_rn(m2c12, n3, c6));
                    } else {
                        const float2 c12x2 = make_float2(2.f * tp.x, 2.f * tp.x);
                        const float2 dsq = __fmul2_rn(d2, d2);
                        const float2 d6 = __fmul2_rn(dsq, d2);
                        float r0, r1;
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(-d6.x));
                        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(-d6.y));
                        float2 n3 = make_float2(r0, r1);
                        if (NEWTON) n3 = __ffma2_rn(n3, __ffma2_rn(d6, n3, one2), n3);
                        float2 n3m = n3;
                        if (MASK) {
                            const float2 m =
                                make_float2(set_lt(d2.x, g.rc2f), set_lt(d2.y, g.rc2f));
                            n3m = __fmul2_rn(n3, m);
                            fe[j] = __ffma2_rn(m, sh, fe[j]);
                        }
                        fe[j] = __ffma2_rn(n3m, __ffma2_rn(c12, n3m, c6), fe[j]);
                        const float2 ea = __fmul2_rn(n3m, __ffma2_rn(c12x2, n3m, c6));
                        fp = __fmul2_rn(ea, __fmul2_rn(n3, dsq));
                    }
                    fh[j][q][0] = __ffma2_rn(fp, dx2, fh[j][q][0]);
                    fh[j][q][1] = __ffma2_rn(fp, dy2, fh[j][q][1]);
                    fh[j][q][2] = __ffma2_rn(fp, dz2, fh[j][q][2]);
                    if (SYM)   // F_0 - F_1 in ff[j][0]
                        ff[j][0] = q ? __ffma2_rn(fp, make_float2(-1.f, -1.f), ff[j][0])
                                     : __fadd2_rn(fp, ff[j][0]);
                    else
                        ff[j][q] = __fadd2_rn(fp, ff[j][q]);
                }
            }
        }
        if (!MASK) shift_sum += (double)fs;
#pragma unroll
        for (int j = 0; j < PP; ++j) {
            acc[2 * j].e += (double)fe[j].x;
            acc[2 * j + 1].e += (double)fe[j].y;
        }
        }
        if constexpr (GSUM_NT > 0) {
#pragma unroll
            for (int j = 0; j < PP; ++j)
#pragma unroll
                for (int l = 0; l < 2; ++l)
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            grad_slot<GSUM_NT>(gsum, 2 * j + l, 3 * q + k) +=
                                (double)(l ? fh[j][q][k].y : fh[j][q][k].x);
                        if (!SYM || q == 0)
                            grad_slot<GSUM_NT>(gsum, 2 * j + l, 6 + q) +=
                                (double)(l ? ff[j][q].y : ff[j][q].x);
                    }
        } else {
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                AdjAcc &a0 = acc[2 * j], &a1 = acc[2 * j + 1];
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    if (!SYM || q == 0) {
                        a0.f[q] += (double)ff[j][q].x;
                        a1.f[q] += (double)ff[j][q].y;
                    }
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        a0.h[q][k] += (double)fh[j][q][k].x;
                        a1.h[q][k] += (double)fh[j][q][k].y;
                    }
                }
            }
        }
    }
}

// Outer shell entries (RegionInfo::n_outer: beyond rc + rho + 1e-3 A of the
// region origin, so |d0| > rc for every pose center of the region), symmetric
// sites only.  With q_s = k0 + m_s t and m_1 = -m_0, a director's site on the
// entry's side (m_s t <= 0) has q = k0 - |m_0| |t| and the other q >= k0 =
// |d0|^2 + o^2 > rc^2: at most the near one is inside.  Only that one is
// evaluated, with the operations of far_chunk_adj (fma(-|m0|, |t|, k0) is
// the near site's fma(m_s, t, k0) bit for bit); the other is out in FP32
// (its q is at least k0, which exceeds rc^2 by 0.025 A^2 and more) as in
// FP64, so shell_border_repair sees the decisions this loop took.  Gradient
// partials: A = sum fp d0, B = sum sigma fp d0, C = sum sigma fp (sigma = +1
// where the near site is site 0, -1 where it is site 1), flushed as H_0 =
// (A + B) / 2, H_1 = (A - B) / 2 and F_0 - F_1 = C (f[0] of the symmetric
// loops).  BORDER 2: the per-director cutoff-border test of far_chunk_adj.
template <int P, int FLUSH, int UNROLL, int GSUM_NT, int BORDER>
__device__ __forceinline__ void far_chunk_outer(const float4 *hb, const float4 *stf, int len,
                                                const FarGeom &g, const float2 (&ux)[P / 2],
                                                const float2 (&uy)[P / 2],
                                                const float2 (&uz)[P / 2], AdjAcc (&acc)[P],
                                                double *gsum = nullptr,
                                                float *border = nullptr) {
    static_assert(BORDER != 1, "the outer loop serves the symmetric-site kernels");
    constexpr int PP = P / 2;
    const float2 nam = make_float2(-fabsf(g.m0.x), -fabsf(g.m0.x));   // -|m0|
    const bool m0neg = g.m0.x < 0.f;   // site 0 is the near one where t > 0
#pragma unroll 1
    for (int e0 = 0; e0 < len; e0 += FLUSH) {
        float2 fa[PP][3], fb[PP][3], fc[PP];
#pragma unroll
        for (int j = 0; j < PP; ++j) {
            fc[j] = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < 3; ++k) fa[j][k] = fb[j][k] = make_float2(0.f, 0.f);
        }
        const int e1 = min(e0 + FLUSH, len);
#pragma unroll 1
        for (int b0 = e0; b0 < e1; b0 += 16) {   // energy partials: 16 entries
            float2 fe[PP];
#pragma unroll
            for (int j = 0; j < PP; ++j) fe[j] = make_float2(0.f, 0.f);
            const int b1 = min(b0 + 16, e1);
#pragma unroll UNROLL
            for (int e = b0; e < b1; ++e) {
                float2 k0, dx2, dy2, dz2, c12, c6, sh, mc6, m2c12;
                float ts = 0.f;
                {
                    const float4 h = hb[e];
                    const float4 tp = stf[__float_as_int(h.w)];   // (c12, c6, shift, -)
                    const float dx = h.x - g.cx, dy = h.y - g.cy, dz = h.z - g.cz;
                    const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    if (dd > g.out2) continue;
                    k0 = make_float2(dd + g.oo0, dd + g.oo0);
                    dx2 = make_float2(dx, dx);
                    dy2 = make_float2(dy, dy);
                    dz2 = make_float2(dz, dz);
                    c12 = make_float2(tp.x, tp.x);
                    c6 = make_float2(tp.y, tp.y);
                    sh = make_float2(tp.z, tp.z);
                    mc6 = make_float2(-tp.y, -tp.y);
                    m2c12 = make_float2(-2.f * tp.x, -2.f * tp.x);
                    if (BORDER == 2) ts = fabsf(fmaf(dd, g.inv2o, g.tb));
                }
#pragma unroll
                for (int j = 0; j < PP; ++j) {
                    const float2 t =
                        __ffma2_rn(dx2, ux[j], __ffma2_rn(dy2, uy[j], __fmul2_rn(dz2, uz[j])));
                    const float2 at = make_float2(fabsf(t.x), fabsf(t.y));
                    if (BORDER == 2) {
                        border[2 * j] = fminf(border[2 * j], fabsf(at.x - ts));
                        border[2 * j + 1] = fminf(border[2 * j + 1], fabsf(at.y - ts));
                    }
                    const float2 d2 = __ffma2_rn(nam, at, k0);
                    float r0, r1;
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(d2.x));
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(d2.y));
                    const float2 n1 = make_float2(r0, r1);
                    float2 n3 = __fmul2_rn(__fmul2_rn(n1, n1), n1);
                    const float2 m = make_float2(set_lt(d2.x, g.rc2f), set_lt(d2.y, g.rc2f));
                    n3 = __fmul2_rn(n3, m);
                    fe[j] = __ffma2_rn(m, sh, fe[j]);
                    fe[j] = __ffma2_rn(n3, __ffma2_rn(c12, n3, mc6), fe[j]);
                    const float2 fp = __fmul2_rn(__fmul2_rn(n1, n3), __ffma2_rn(m2c12, n3, c6));
                    const float2 sfp = make_float2((t.x > 0.f) == m0neg ? fp.x : -fp.x,
                                                   (t.y > 0.f) == m0neg ? fp.y : -fp.y);
                    fa[j][0] = __ffma2_rn(fp, dx2, fa[j][0]);
                    fa[j][1] = __ffma2_rn(fp, dy2, fa[j][1]);
                    fa[j][2] = __ffma2_rn(fp, dz2, fa[j][2]);
                    fb[j][0] = __ffma2_rn(sfp, dx2, fb[j][0]);
                    fb[j][1] = __ffma2_rn(sfp, dy2, fb[j][1]);
                    fb[j][2] = __ffma2_rn(sfp, dz2, fb[j][2]);
                    fc[j] = __fadd2_rn(sfp, fc[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                acc[2 * j].e += (double)fe[j].x;
                acc[2 * j + 1].e += (double)fe[j].y;
            }
        }
#pragma unroll
        for (int j = 0; j < PP; ++j)
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                const int p = 2 * j + l;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double a = (double)(l ? fa[j][k].y : fa[j][k].x);
                    const double b = (double)(l ? fb[j][k].y : fb[j][k].x);
                    if constexpr (GSUM_NT > 0) {
                        grad_slot<GSUM_NT>(gsum, p, k) += 0.5 * (a + b);
                        grad_slot<GSUM_NT>(gsum, p, 3 + k) += 0.5 * (a - b);
                    } else {
                        acc[p].h[0][k] += 0.5 * (a + b);
                        acc[p].h[1][k] += 0.5 * (a - b);
                    }
                }
                const double c = (double)(l ? fc[j].y : fc[j].x);
                if constexpr (GSUM_NT > 0)
                    grad_slot<GSUM_NT>(gsum, p, 6) += c;
                else
                    acc[p].f[0] += c;
            }
    }
}

}  // namespace vext
