// Pose energies and the analytic adjoint for arbitrary poses (String images,
// random pose batches, the torch autograd path).
//
// Poses are wrapped into the cell (FP64) and binned on a fractional grid of
// ~0.75 A bins; every bin is a region with its own list (built once per
// system, system.cu).  One CTA = one work item (a bin and up to kPoseThreads
// of its poses, one pose per thread; warps without a pose skip the pair
// loops).  Pair terms are recomputed, never stored:
//   E   = sum  c12 i6^2 - c6 i6 + shift                 (d2 < rc^2)
//   dE/dr_site = sum i2 i6 (6 c6 - 12 c12 i6) (r_site - x)  (floor2 < d2 < rc^2)
// (inside the contact floor the energy is constant, so its gradient is 0).
// dE/dcenter = F0 + F1, dE/du = o0 F0 + o1 F1, and dE/dq = J(q)^T dE/du
// projected onto the tangent space of the unit quaternion sphere, with
// u = R(q) e_x = (1 - 2(y^2 + z^2), 2(xy + wz), 2(xz - wy)).
// Precision follows the field kernel: near chunks FP64, far chunks FP32 with
// periodic FP64 flushes, FP64 re-evaluation of poses in the refinement band
// and of poses with a shell pair within kBorderTol of the cutoff (where the
// FP32 and FP64 cutoff tests may disagree).
#include <algorithm>
#include <cmath>

#include "pair.cuh"

namespace vext {

constexpr int kPoseThreads = 128;   // poses per work item: the CTA width


struct PoseArgs {
    Mat3 H, Hinv;
    double rc2;
    float rc2f;
    double off0, off1;
    int n;
    const double *centers;   // [n][3] Cartesian
    const double *quats;     // [n][4]
    double *wf;              // [n][3] wrapped fractional
    double *u;               // [n][3] director
    int *bin;                // [n]
    int nb0, nb1, nb2, n_bins;
    int *counts, *starts, *cursor;   // [n_bins], [n_bins + 1], [n_bins]
    int *order;              // [n] pose ids sorted by bin
    int *items;              // [0] = count, then (bin, first, len)
    int max_items;
    int item_poses;          // poses per work item (the CTA width)
    double floor_out2;       // site-atom d2 above which no type's contact floor applies
    const RegionInfo *regs;
    const float4 *hi, *lo;
    const float4 *tf;
    const double *td;
    int n_types;
    double *energy, *gc, *gq, *gu;
    int *refine;             // [0] = count, then pose ids
    double band_lo, band_hi;
    int *status;
};



__global__ void pose_prep_kernel(PoseArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const double *q = a.quats + 4 * p;
    const double nq = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const double w = q[0] / nq, x = q[1] / nq, y = q[2] / nq, z = q[3] / nq;
    a.u[3 * p + 0] = 1.0 - 2.0 * (y * y + z * z);
    a.u[3 * p + 1] = 2.0 * (x * y + w * z);
    a.u[3 * p + 2] = 2.0 * (x * z - w * y);
    const double c0 = a.centers[3 * p], c1 = a.centers[3 * p + 1], c2 = a.centers[3 * p + 2];
    int b[3];
    const int nb[3] = {a.nb0, a.nb1, a.nb2};
    bool ok = isfinite(nq) && nq > 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double v = c0 * a.Hinv.m[k] + c1 * a.Hinv.m[3 + k] + c2 * a.Hinv.m[6 + k];
        ok = ok && isfinite(v);
        v = isfinite(v) ? v - floor(v) : 0.0;
        if (v >= 1.0) v = 0.0;
        b[k] = min(nb[k] - 1, (int)(v * nb[k]));
        a.wf[3 * p + k] = v;
    }
    if (!ok) atomicExch(a.status, DEV_BAD_INPUT);
    const int id = (b[0] * a.nb1 + b[1]) * a.nb2 + b[2];
    a.bin[p] = id;
    atomicAdd(&a.counts[id], 1);
}

// Single CTA: bin starts and the (bin, first, len) work items.
__global__ void pose_scan_kernel(PoseArgs a) {
    __shared__ int carry[2];
    __shared__ int warp_tot[2][32];
    if (threadIdx.x == 0) carry[0] = carry[1] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < a.n_bins; base += blockDim.x) {
        const int b = base + threadIdx.x;
        const int cnt = b < a.n_bins ? a.counts[b] : 0;
        const int nit = (cnt + a.item_poses - 1) / a.item_poses;
        int xc = cnt, xi = nit;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int yc = __shfl_up_sync(0xffffffffu, xc, o), yi = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) {
                xc += yc;
                xi += yi;
            }
        }
        if (lane == 31) {
            warp_tot[0][warp] = xc;
            warp_tot[1][warp] = xi;
        }
        __syncthreads();
        int wc = 0, wi = 0;
        for (int w = 0; w < warp; ++w) {
            wc += warp_tot[0][w];
            wi += warp_tot[1][w];
        }
        const int pc = carry[0] + wc + xc - cnt, pi = carry[1] + wi + xi - nit;
        if (b < a.n_bins) {
            a.starts[b] = pc;
            for (int k = 0; k < nit; ++k) {
                const int it = pi + k;
                if (it < a.max_items) {
                    a.items[1 + 3 * it] = b;
                    a.items[2 + 3 * it] = pc + k * a.item_poses;
                    a.items[3 + 3 * it] = min(a.item_poses, cnt - k * a.item_poses);
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tc = 0, ti = 0;
            for (int w = 0; w < nw; ++w) {
                tc += warp_tot[0][w];
                ti += warp_tot[1][w];
            }
            carry[0] += tc;
            carry[1] += ti;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.starts[a.n_bins] = carry[0];
        a.items[0] = min(carry[1], a.max_items);
    }
}

__global__ void pose_scatter_kernel(PoseArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int b = a.bin[p];
    a.order[a.starts[b] + atomicAdd(&a.cursor[b], 1)] = p;
}

// Outputs of pose p from its energy, dE/dcenter (gc3) and dE/du (gu3, not
// projected): dE/dq = J(q)^T dE/du, projected on the tangent space of |q| = 1.
__device__ __forceinline__ void write_pose_sums(const PoseArgs &a, int p, double e,
                                                const double *gc3, const double *gu) {
    if (a.energy) a.energy[p] = e;
    if (a.gc)
        for (int k = 0; k < 3; ++k) a.gc[3 * p + k] = gc3[k];
    if (a.gu)
        for (int k = 0; k < 3; ++k) a.gu[3 * p + k] = gu[k];
    if (a.gq) {
        const double *q = a.quats + 4 * p;
        const double nq = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        const double w = q[0] / nq, x = q[1] / nq, y = q[2] / nq, z = q[3] / nq;
        double g[4];
        g[0] = 2 * z * gu[1] - 2 * y * gu[2];
        g[1] = 2 * y * gu[1] + 2 * z * gu[2];
        g[2] = -4 * y * gu[0] + 2 * x * gu[1] - 2 * w * gu[2];
        g[3] = -4 * z * gu[0] + 2 * w * gu[1] + 2 * x * gu[2];
        const double dot = g[0] * w + g[1] * x + g[2] * y + g[3] * z;
        a.gq[4 * p + 0] = (g[0] - dot * w) / nq;
        a.gq[4 * p + 1] = (g[1] - dot * x) / nq;
        a.gq[4 * p + 2] = (g[2] - dot * y) / nq;
        a.gq[4 * p + 3] = (g[3] - dot * z) / nq;
    }
}

// The same from the two site forces F0, F1 (dE/dcenter = F0 + F1, dE/du =
// o0 F0 + o1 F1).
__device__ __forceinline__ void write_pose(const PoseArgs &a, int p, double e, const double *F0,
                                           const double *F1) {
    double gc[3], gu[3];
    for (int k = 0; k < 3; ++k) {
        gc[k] = F0[k] + F1[k];
        gu[k] = a.off0 * F0[k] + a.off1 * F1[k];
    }
    write_pose_sums(a, p, e, gc, gu);
}

// Far entries [e_begin, e_end) of one staged chunk for one pose: the packed
// FP32x2 loop of the field kernels with the lanes holding the pose's two
// sites.  Per lane d = x - r_s, n1 = hardware reciprocal of d2, n3 = n1^3,
// e = n3 (c12 n3 - c6), fp = (n1 n3)(c6 - 2 c12 n3) = (dE/dd2) / 3 and
// G_s += fp d, so that dE/dr_s = -6 G_s.  Far entries lie beyond r_split of
// every site of every pose of the bin, so the contact floor never applies.
// MASK = false for inner entries (inside the cutoff of every such site): no
// cutoff mask, and the shift is summed once per entry into shift_sum (added
// to both sites).  Energy partials are flushed into FP64 every 16 entries,
// the gradient partials once per call.  MASK: bmin (per site) receives the
// smallest |d2 - rc^2| met, for the FP64 re-evaluation of poses with a pair
// too close to the cutoff for the FP32 test (kBorderTol).
template <bool MASK>
__device__ __forceinline__ void pose_far(const float4 *hb, const float4 *stf, int e_begin,
                                         int e_end, float2 nsx, float2 nsy, float2 nsz,
                                         float rc2f, double (&E)[2], double (&F)[2][3],
                                         double &shift_sum, float2 &bmin) {
    float2 gx = make_float2(0.f, 0.f), gy = gx, gz = gx;
#pragma unroll 1
    for (int e0 = e_begin; e0 < e_end; e0 += 16) {
        float2 fe = make_float2(0.f, 0.f);
        float fs = 0.f;
        const int e1 = min(e0 + 16, e_end);
#pragma unroll 2
        for (int e = e0; e < e1; ++e) {
            float2 dx, dy, dz, c12, mc6, m2c12, c6, sh;
            {
                const float4 h = hb[e];
                const float4 tp = stf[__float_as_int(h.w)];   // (c12, c6, shift, floor2)
                dx = __fadd2_rn(make_float2(h.x, h.x), nsx);
                dy = __fadd2_rn(make_float2(h.y, h.y), nsy);
                dz = __fadd2_rn(make_float2(h.z, h.z), nsz);
                c12 = make_float2(tp.x, tp.x);
                mc6 = make_float2(-tp.y, -tp.y);
                m2c12 = make_float2(-2.f * tp.x, -2.f * tp.x);
                c6 = make_float2(tp.y, tp.y);
                sh = make_float2(tp.z, tp.z);
                if (!MASK) fs += tp.z;
            }
            const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            float r0, r1;
            asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(d2.x));
            asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(d2.y));
            const float2 n1 = make_float2(r0, r1);
            float2 n3 = __fmul2_rn(__fmul2_rn(n1, n1), n1);
            if (MASK) {
                const float2 m = make_float2(set_lt(d2.x, rc2f), set_lt(d2.y, rc2f));
                n3 = __fmul2_rn(n3, m);
                fe = __ffma2_rn(m, sh, fe);
                const float2 x = __fadd2_rn(d2, make_float2(-rc2f, -rc2f));
                bmin.x = fminf(bmin.x, fabsf(x.x));
                bmin.y = fminf(bmin.y, fabsf(x.y));
            }
            fe = __ffma2_rn(n3, __ffma2_rn(c12, n3, mc6), fe);
            const float2 fp = __fmul2_rn(__fmul2_rn(n1, n3), __ffma2_rn(m2c12, n3, c6));
            gx = __ffma2_rn(fp, dx, gx);
            gy = __ffma2_rn(fp, dy, gy);
            gz = __ffma2_rn(fp, dz, gz);
        }
        E[0] += (double)fe.x;
        E[1] += (double)fe.y;
        if (!MASK) shift_sum += (double)fs;
    }
    F[0][0] -= 6.0 * (double)gx.x;
    F[1][0] -= 6.0 * (double)gx.y;
    F[0][1] -= 6.0 * (double)gy.x;
    F[1][1] -= 6.0 * (double)gy.y;
    F[0][2] -= 6.0 * (double)gz.x;
    F[1][2] -= 6.0 * (double)gz.y;
}

// MIXED: near pairs take the FP64 reciprocal as a hardware seed + one Newton
// step (relative error <= 2^-46) and far pairs the packed FP32 loop; otherwise
// (the FP64 mode: every entry is near) the correctly rounded reciprocal.
// NEAR_IN: the host proved every near pair inside the cutoff (r_split + 2
// (rho + max|offset|) < rc), so near pairs skip the cutoff test.
template <int NT, bool MIXED, bool NEAR_IN>
__global__ void __launch_bounds__(NT) pose_kernel(PoseArgs a) {
    const int item = blockIdx.x;
    if (item >= a.items[0]) return;   // uniform over the CTA
    extern __shared__ __align__(128) unsigned char smem[];
    Stager st;
    st.bar = reinterpret_cast<uint64_t *>(smem);
    st.hib = reinterpret_cast<float4 *>(smem + 64);
    st.lob = st.hib + kStages * kCH;
    double *ed = reinterpret_cast<double *>(st.lob + kStages * kCH);
    float4 *stf = reinterpret_cast<float4 *>(ed + 4 * kCH);
    double *std4 = reinterpret_cast<double *>(stf + a.n_types);

    const int tid = threadIdx.x;
    const int bin = a.items[1 + 3 * item], first = a.items[2 + 3 * item],
              len_p = a.items[3 + 3 * item];
    const RegionInfo r = a.regs[bin];
    ChunkPlan plan;
    plan.init(r);
    for (int t = tid; t < a.n_types; t += NT) {
        stf[t] = a.tf[t];
#pragma unroll
        for (int k = 0; k < 4; ++k) std4[4 * t + k] = a.td[4 * t + k];
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&st.bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int c = 0; c < min(kStages, plan.n_chunks); ++c) st.issue(plan, a.hi, a.lo, c, c);

    const bool valid = tid < len_p;
    const bool warp_on = (tid & ~31) < len_p;   // uniform over the warp
    const int p = a.order[first + (valid ? tid : 0)];
    double cx, cy, cz;
    frac_to_cart(a.H, a.wf[3 * p] - r.of[0], a.wf[3 * p + 1] - r.of[1], a.wf[3 * p + 2] - r.of[2],
                 cx, cy, cz);
    const double ux = a.u[3 * p], uy = a.u[3 * p + 1], uz = a.u[3 * p + 2];
    double sd[2][3];
    double E[2] = {0, 0}, F[2][3] = {{0, 0, 0}, {0, 0, 0}}, shift_sum = 0.0;
    float2 bmin = make_float2(__int_as_float(0x7f800000), __int_as_float(0x7f800000));
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const double off = s ? a.off1 : a.off0;
        sd[s][0] = cx + off * ux;
        sd[s][1] = cy + off * uy;
        sd[s][2] = cz + off * uz;
    }
    // the sites negated, one per lane, for the far loop's d = x - r_s
    const float2 nsx = make_float2(-(float)sd[0][0], -(float)sd[1][0]),
                 nsy = make_float2(-(float)sd[0][1], -(float)sd[1][1]),
                 nsz = make_float2(-(float)sd[0][2], -(float)sd[1][2]);

    for (int c = 0; c < plan.n_chunks; ++c) {
        const int s = c % kStages;
        const bool ok = mbar_wait_bounded(&st.bar[s], (c / kStages) & 1, a.status);
        if (!__syncthreads_and(ok)) {
            if (tid == 0)
                for (int cc = c; cc < min(c + kStages, plan.n_chunks); ++cc)
                    mbar_drain(&st.bar[cc % kStages], (cc / kStages) & 1);
            return;
        }
        int start, len;
        bool near;
        plan.chunk(c, start, len, near);
        if (near) {
            const float4 *hb = st.hib + s * kCH, *lb = st.lob + s * kCH;
            for (int e = tid; e < len; e += NT) {
                const float4 h = hb[e], l = lb[e];
                ed[4 * e + 0] = (double)h.x + (double)l.x;
                ed[4 * e + 1] = (double)h.y + (double)l.y;
                ed[4 * e + 2] = (double)h.z + (double)l.z;
                ed[4 * e + 3] = (double)__float_as_int(h.w);
            }
            __syncthreads();
            if (warp_on) {
                const double2 *ed2 = reinterpret_cast<const double2 *>(ed);
                const double2 *td2 = reinterpret_cast<const double2 *>(std4);
#pragma unroll 1
                for (int e = 0; e < len; ++e) {
                    const double2 xy = ed2[2 * e], zt = ed2[2 * e + 1];
                    const int t = (int)zt.y;
                    const double2 cc = td2[2 * t], sh = td2[2 * t + 1];
                    const double a12 = -12.0 * cc.x, a6 = 6.0 * cc.y;
                    double dx[2], dy[2], dz[2], d2[2];
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        dx[q] = sd[q][0] - xy.x;
                        dy[q] = sd[q][1] - xy.y;
                        dz[q] = sd[q][2] - zt.x;
                        d2[q] = fma(dx[q], dx[q], fma(dy[q], dy[q], dz[q] * dz[q]));
                    }
                    if (MIXED && NEAR_IN && fmin(d2[0], d2[1]) > a.floor_out2) {
                        // every pair inside the cutoff and clear of the floor:
                        // no tests, the shift summed once per entry
                        shift_sum += sh.x;
#pragma unroll
                        for (int q = 0; q < 2; ++q) {
                            const double i2 = rcp64_nr<1>(d2[q]);
                            const double i6 = i2 * i2 * i2;
                            E[q] = fma(i6, fma(cc.x, i6, -cc.y), E[q]);
                            const double w = i2 * i6 * fma(a12, i6, a6);
                            F[q][0] = fma(w, dx[q], F[q][0]);
                            F[q][1] = fma(w, dy[q], F[q][1]);
                            F[q][2] = fma(w, dz[q], F[q][2]);
                        }
                        continue;
                    }
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const double s2 = fmax(d2[q], sh.y);
                        const double i2 = MIXED ? rcp64_nr<1>(s2) : __drcp_rn(s2);
                        const double i6 = i2 * i2 * i2;
                        const double en = fma(i6, fma(cc.x, i6, -cc.y), sh.x);
                        const bool in = NEAR_IN || d2[q] < a.rc2;
                        const double w = (in && d2[q] > sh.y) ? i2 * i6 * fma(a12, i6, a6) : 0.0;
                        E[q] += in ? en : 0.0;
                        F[q][0] = fma(w, dx[q], F[q][0]);
                        F[q][1] = fma(w, dy[q], F[q][1]);
                        F[q][2] = fma(w, dz[q], F[q][2]);
                    }
                }
            }
        } else if (MIXED) {
            // inner entries first, then the shell (the chunk may straddle them)
            const float4 *hb = st.hib + s * kCH;
            const int split = min(max(r.n_near + r.n_inner - start, 0), len);
            if (warp_on) {
                pose_far<false>(hb, stf, 0, split, nsx, nsy, nsz, a.rc2f, E, F, shift_sum, bmin);
                pose_far<true>(hb, stf, split, len, nsx, nsy, nsz, a.rc2f, E, F, shift_sum, bmin);
            }
        }
        __syncthreads();
        if (tid == 0 && c + kStages < plan.n_chunks)
            st.issue(plan, a.hi, a.lo, c + kStages, c + kStages);
    }
    if (valid) {
        const double e = E[0] + E[1] + 2.0 * shift_sum;
        write_pose(a, p, e, F[0], F[1]);
        // the refinement band, or a shell pair within kBorderTol of the cutoff
        if (a.refine && ((e > a.band_lo && e < a.band_hi) || fminf(bmin.x, bmin.y) < kBorderTol)) {
            const int k = atomicAdd(&a.refine[0], 1);
            a.refine[1 + k] = p;
        }
    }
}

// FP64 re-evaluation of flagged poses, one warp per pose: the pair test and
// terms of the FP64 pose sums (fp64_pose_pairs_both: both sites per entry,
// the reciprocal from the hardware seed and two Newton steps), the lanes
// striding over the bin's list.
__global__ void pose_refine_kernel(PoseArgs a) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int count = a.refine[0];
    for (int q = warp; q < count; q += nwarps) {
        const int p = a.refine[1 + q];
        const RegionInfo r = a.regs[a.bin[p]];
        double cx, cy, cz;
        frac_to_cart(a.H, a.wf[3 * p] - r.of[0], a.wf[3 * p + 1] - r.of[1],
                     a.wf[3 * p + 2] - r.of[2], cx, cy, cz);
        const double u[3] = {a.u[3 * p], a.u[3 * p + 1], a.u[3 * p + 2]};
        double e = 0.0, g[6];
        fp64_pose_pairs_both(a.hi, a.lo, a.td, r.off, r.n_total, lane, 32, a.rc2, a.off0, a.off1,
                             cx, cy, cz, u, e, g);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, o);
#pragma unroll
            for (int k = 0; k < 6; ++k) g[k] += __shfl_xor_sync(0xffffffffu, g[k], o);
        }
        if (lane == 0) write_pose_sums(a, p, e, g, g + 3);
    }
}

// ---------------------------------------------------------------- host side

struct Bump {
    char *base;
    size_t used = 0;
    template <typename T>
    T *take(size_t n) {
        used = (used + 255) & ~(size_t)255;
        T *p = reinterpret_cast<T *>(base + used);
        used += n * sizeof(T);
        return p;
    }
};

static size_t pose_scratch_bytes(int n, int n_bins, int max_items, bool host_io) {
    size_t b = 0;
    auto add = [&](size_t bytes) { b = ((b + 255) & ~(size_t)255) + bytes; };
    add(sizeof(double) * 3 * n);          // wf
    add(sizeof(double) * 3 * n);          // u
    add(sizeof(int) * n);                 // bin
    add(sizeof(int) * n);                 // order
    add(sizeof(int) * n_bins);            // counts
    add(sizeof(int) * (n_bins + 1));      // starts
    add(sizeof(int) * n_bins);            // cursor
    add(sizeof(int) * (1 + 3 * (size_t)max_items));
    add(sizeof(int) * (n + 1));           // refine
    add(sizeof(double) * n);              // energy (when the caller passes none)
    if (host_io) {
        add(sizeof(double) * 3 * n);      // centers
        add(sizeof(double) * 4 * n);      // quats
        add(sizeof(double) * 3 * n);      // gc
        add(sizeof(double) * 4 * n);      // gq
        add(sizeof(double) * 3 * n);      // gu
    }
    return b + 256;
}

// Enqueue the whole pose pipeline on `st` (device pointers, no host
// synchronisation once the bin lists exist; safe inside stream capture after
// a first call has built the lists and the scratch).  Energies go to `energy`
// (a scratch buffer when NULL).
int pose_enqueue(System *sys, int n, const double *centers, const double *quats,
                 const Options &o, double *energy, double *gc, double *gq, double *gu,
                 cudaStream_t st) {
    if (n < 0) return fail(VEXT_ERR_ARGUMENT, "negative pose count");
    if (n == 0) return 0;
    if (!centers || !quats) return fail(VEXT_ERR_ARGUMENT, "centers and quaternions required");
    if (o.mode != VEXT_MODE_MIXED && o.mode != VEXT_MODE_FP64)
        return fail(VEXT_ERR_ARGUMENT, "unknown precision mode %d", o.mode);
    const double r_split = o.mode == VEXT_MODE_FP64 ? 1e30 : o.r_split;
    RegionSet *rs = nullptr;
    VEXT_TRY(get_bin_regions(sys, r_split, &rs, st));
    const int n_bins = rs->n_regions;
    // Fewer than 64 poses per bin on average: the binned pipeline would give
    // most of its per-bin CTAs a handful of poses for a whole list each; one
    // to eight warps per pose are faster there (String paths, small batches).
    if ((long long)n < 64LL * n_bins)
        return pose_warp_enqueue(sys, rs, n, centers, quats, o,
                                 energy ? energy : nullptr, gc, gq, gu, st);
    const int item_poses = kPoseThreads;
    const int max_items = n_bins + (n + item_poses - 1) / item_poses;
    const size_t bytes = pose_scratch_bytes(n, n_bins, max_items, false);
    VEXT_TRY(ensure_capacity(*reinterpret_cast<char **>(&sys->d_pose_scratch),
                             sys->pose_scratch_cap, bytes));
    Bump bump{reinterpret_cast<char *>(sys->d_pose_scratch)};
    PoseArgs a;
    a.H = sys->H;
    a.Hinv = sys->Hinv;
    a.rc2 = sys->cutoff * sys->cutoff;
    a.rc2f = (float)a.rc2;
    a.off0 = sys->offsets[0];
    a.off1 = sys->offsets[1];
    a.n = n;
    a.wf = bump.take<double>(3 * (size_t)n);
    a.u = bump.take<double>(3 * (size_t)n);
    a.bin = bump.take<int>(n);
    a.order = bump.take<int>(n);
    a.nb0 = rs->nb[0];
    a.nb1 = rs->nb[1];
    a.nb2 = rs->nb[2];
    a.n_bins = n_bins;
    a.counts = bump.take<int>(n_bins);
    a.starts = bump.take<int>(n_bins + 1);
    a.cursor = bump.take<int>(n_bins);
    a.items = bump.take<int>(1 + 3 * (size_t)max_items);
    a.max_items = max_items;
    a.item_poses = item_poses;
    {
        // beyond sqrt(max floor2) (plus a relative margin far above FP64
        // rounding) no pair of any type is inside its contact floor
        double fl = 0.0;
        for (int t = 0; t < sys->n_types; ++t) fl = std::max(fl, sys->h_td[4 * t + 3]);
        const double rf = std::sqrt(fl) * (1.0 + 1e-9) + 1e-9;
        a.floor_out2 = rf * rf;
    }
    a.regs = rs->d_info;
    a.hi = rs->d_hi;
    a.lo = rs->d_lo;
    a.tf = sys->d_tf;
    a.td = sys->d_td;
    a.n_types = sys->n_types;
    const bool refine = o.mode == VEXT_MODE_MIXED;   // band and border poses
    int *d_refine = bump.take<int>((size_t)n + 1);
    a.refine = refine ? d_refine : nullptr;
    a.band_lo = o.band_lo;
    a.band_hi = o.band_hi;
    a.status = sys->d_status;
    double *e_tmp = bump.take<double>(n);
    a.centers = centers;
    a.quats = quats;
    a.energy = energy ? energy : e_tmp;
    a.gc = gc;
    a.gq = gq;
    a.gu = gu;
    VEXT_CUDA(cudaMemsetAsync(a.counts, 0, sizeof(int) * n_bins, st));
    VEXT_CUDA(cudaMemsetAsync(a.cursor, 0, sizeof(int) * n_bins, st));
    VEXT_CUDA(cudaMemsetAsync(d_refine, 0, sizeof(int), st));
    const int pb = (n + 255) / 256;
    pose_prep_kernel<<<pb, 256, 0, st>>>(a);
    VEXT_CUDA(cudaGetLastError());
    pose_scan_kernel<<<1, 1024, 0, st>>>(a);
    VEXT_CUDA(cudaGetLastError());
    pose_scatter_kernel<<<pb, 256, 0, st>>>(a);
    VEXT_CUDA(cudaGetLastError());
    const size_t smem = kStageBytes + (size_t)kCH * 4 * sizeof(double) + (size_t)a.n_types * 48;
    double rho = 0;
    for (const RegionInfo &r : rs->h_info) rho = std::max(rho, r.rho);
    const bool near_in = o.mode == VEXT_MODE_MIXED &&
                         r_split + 2.0 * (rho + sys->max_offset) + 1e-6 < sys->cutoff;
    auto kernel = o.mode != VEXT_MODE_MIXED ? pose_kernel<kPoseThreads, false, false>
                  : near_in                 ? pose_kernel<kPoseThreads, true, true>
                                            : pose_kernel<kPoseThreads, true, false>;
    VEXT_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kernel<<<max_items, item_poses, smem, st>>>(a);
    VEXT_CUDA(cudaGetLastError());
    if (refine) {
        pose_refine_kernel<<<std::min(1184, (n + 7) / 8), 256, 0, st>>>(a);
        VEXT_CUDA(cudaGetLastError());
    }
    return 0;
}

// Host-pointer wrapper: copies in, pose_enqueue, copies out, status check.
static int pose_run_host(System *sys, int n, const double *centers, const double *quats,
                         const Options &o, double *energy, double *gc, double *gq, double *gu,
                         cudaStream_t st) {
    if (n < 0) return fail(VEXT_ERR_ARGUMENT, "negative pose count");
    if (n == 0) return 0;
    if (!centers || !quats) return fail(VEXT_ERR_ARGUMENT, "centers and quaternions required");
    const size_t per = sizeof(double) * (size_t)n;
    VEXT_TRY(ensure_capacity(sys->d_pose_io, sys->pose_io_cap, 18 * (size_t)n));
    double *dc = sys->d_pose_io, *dq = dc + 3 * (size_t)n, *de = dq + 4 * (size_t)n,
           *dgc = de + n, *dgq = dgc + 3 * (size_t)n, *dgu = dgq + 4 * (size_t)n;
    VEXT_CUDA(cudaMemcpyAsync(dc, centers, 3 * per, cudaMemcpyHostToDevice, st));
    VEXT_CUDA(cudaMemcpyAsync(dq, quats, 4 * per, cudaMemcpyHostToDevice, st));
    VEXT_TRY(pose_enqueue(sys, n, dc, dq, o, de, gc ? dgc : nullptr, gq ? dgq : nullptr,
                          gu ? dgu : nullptr, st));
    if (energy) VEXT_CUDA(cudaMemcpyAsync(energy, de, per, cudaMemcpyDeviceToHost, st));
    if (gc) VEXT_CUDA(cudaMemcpyAsync(gc, dgc, 3 * per, cudaMemcpyDeviceToHost, st));
    if (gq) VEXT_CUDA(cudaMemcpyAsync(gq, dgq, 4 * per, cudaMemcpyDeviceToHost, st));
    if (gu) VEXT_CUDA(cudaMemcpyAsync(gu, dgu, 3 * per, cudaMemcpyDeviceToHost, st));
    return pose_status(sys, st);
}

int pose_status(System *sys, cudaStream_t st) {
    int status = 0;
    VEXT_CUDA(cudaMemcpyAsync(&status, sys->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    VEXT_CUDA(cudaStreamSynchronize(st));
    if (status) {
        VEXT_CUDA(cudaMemsetAsync(sys->d_status, 0, sizeof(int), st));
        VEXT_CUDA(cudaStreamSynchronize(st));
        if (status == DEV_BAD_INPUT)
            return fail(VEXT_ERR_ARGUMENT, "non-finite pose center or zero quaternion");
        return fail(VEXT_ERR_TIMEOUT, "a device wait gave up (status %d)", status);
    }
    return 0;
}

}  // namespace vext

using namespace vext;

extern "C" int vext_pose_energy_grad(vext_system h, int n, const double *centers,
                                     const double *quats, const vext_options *opt, double *energy,
                                     double *grad_center, double *grad_quat,
                                     double *grad_director) {
    if (!h) return fail(VEXT_ERR_ARGUMENT, "null system");
    System *sys = &h->sys;
    std::lock_guard<std::mutex> guard(sys->lock);
    VEXT_CUDA(cudaSetDevice(sys->device));
    return pose_run_host(sys, n, centers, quats, resolve_options(opt), energy, grad_center,
                         grad_quat, grad_director, sys->stream);
}

extern "C" int vext_pose_energy_grad_device(vext_system h, int n, const double *centers,
                                            const double *quats, const vext_options *opt,
                                            double *energy, double *grad_center,
                                            double *grad_quat, double *grad_director,
                                            void *stream) {
    if (!h) return fail(VEXT_ERR_ARGUMENT, "null system");
    System *sys = &h->sys;
    std::lock_guard<std::mutex> guard(sys->lock);
    VEXT_CUDA(cudaSetDevice(sys->device));
    cudaStream_t st = (cudaStream_t)stream;
    VEXT_TRY(pose_enqueue(sys, n, centers, quats, resolve_options(opt), energy, grad_center,
                          grad_quat, grad_director, st));
    return pose_status(sys, st);
}
