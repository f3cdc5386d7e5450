// Batched fields: many systems (frameworks x guests of uneven sizes and cell
// shapes) in ONE persistent launch over a work queue, captured in a CUDA
// graph and replayed.
//
// Work item = (system, region, director block): by default an 8-center
// region x 64 directors (16 x 32 with centers_per_region 16; either way one
// staged list entry serves 512 poses).  Items are sorted by
// estimated cost (list length, longest first) so the tail of the queue is
// made of short items; resident CTAs claim items with one atomicAdd each.
// Each item runs the near (FP64) and the far (packed FP32x2) pair loops of
// pair.cuh back to back on the same staged-chunk pipeline (the mbarrier
// phase sequence continues across items) and writes float32 energies
// straight into the system's [O][S^3] output; poses whose energy falls in the
// refinement band are appended to a list that batch_refine_kernel
// recomputes in FP64.
//
// Autotuning: the CTA shape of the mode's table (128 threads x 4 directors
// or 256 threads x 2, register-resident or shared-memory gradient sums, far
// entry loop unrolled once or twice) and the number of resident CTAs per SM
// are chosen by timing each candidate twice on a strided sample of the queue
// (stride n / (16 x SMs), clamped to 1..128) at creation; the winner is kept
// per (device, kind, size class) so later batches of that class skip the
// timing, and is captured into the graph.  The batch
// keeps pointers to its systems' region lists: the systems must outlive it
// and not be invalidated while it exists.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <tuple>
#include <vector>

#include "pair.cuh"

namespace vext {

struct BatchSys {
    Mat3 H;
    double rc2;
    float rc2f;
    double off0, off1;
    double floor_out2;          // |d0|^2 beyond which no site is inside a contact floor
    int S, O;
    const double *axes;
    const RegionInfo *regs;
    const float4 *hi, *lo;
    const float4 *tf;
    const double *td;
    int n_types;
    int near_mode;              // 1: cutoff test on near pairs, 2: none needed
    int bi, bj, bk, nrj, nrk;   // region grid (pose -> region)
    float *out;                 // [O][S^3]
    float *grad;                // [O][S^3][6] (forward + adjoint batches), else null
    double *out64;              // FP64 copy of the energies [O][S^3], or null
};

// Refinement record flag: the pose is outside the refinement band but has a
// shell pair within kBorderTol of the cutoff; only its shell pairs are
// re-tested (batch_refine_adj_kernel).
constexpr int kRepairOnly = 1 << 30;

// vext_options.variant bit: re-evaluate poses with a shell pair near the
// cutoff in FP64 as a whole instead of repairing their shell pairs (the check
// of the repair)
constexpr int kVariantFullRefine = 4096;

struct BatchArgs {
    const BatchSys *sys;
    const int4 *items;          // (system, region, director block, -)
    int n_items;
    int *counter;
    int *refine;                // [0] count, then (system, pose) pairs
    int refine_cap;
    double band_lo, band_hi;
    int full_refine;            // border poses re-evaluated in FP64 too (kVariantFullRefine)
    int *status;
};

// Forward + adjoint item: the same staged pipeline with the AdjAcc pair loops
// (pair.cuh); writes the energy and [dE/dc, tangent dE/du] of every pose.
// Far entries come in two passes, inner (no cutoff mask, shift summed once
// per entry) and shell, and with OUTER (symmetric sites) a third over the
// outer shell entries, one site per director (far_chunk_outer).
// GSUM: the FP64 gradient sums wait in shared memory (gsum) during the far
// passes, so those passes hold only the energy sums and FP32 partials.
// BORDER 1: border[p] receives the smallest |q - rc^2| (FP32) of director p
// over the masked shell pairs, for the FP64 re-evaluation of poses with a
// pair too close to the cutoff for the FP32 test; 2: the smallest
// | |d0 . u| - |T*| | (symmetric sites), 2 |o| times which is the former.
template <int CB, int G, int P, bool NEWTON, bool RCP1, int UNROLL, int FLUSH, bool GSUM,
          int BORDER, bool OUTER>
__device__ __forceinline__ bool batch_item_adj(const BatchArgs &a, const BatchSys &y,
                                               const RegionInfo &r, Stager &st, double *ed,
                                               const float4 *stf, const double *std4,
                                               double *gsum, unsigned &seq, double cx,
                                               double cy, double cz, int obase, double (&e)[P],
                                               double (&gr)[P][6], float (&border)[P]) {
    constexpr int NT = CB * G, PP = P / 2;
    AdjAcc acc[P];
    adj_zero(acc);
#pragma unroll
    for (int p = 0; p < P; ++p) border[p] = __int_as_float(0x7f800000);   // +inf
    double shift_sum = 0.0;   // inner and near entries: every pair inside the cutoff
    // near pairs (FP64): with GSUM two directors at a time (the near list is
    // staged once per pair; their gradient sums then wait in gsum during the
    // far passes and only the energies stay in registers), else all P in one
    // pass
    // symmetric sites (kernels with the per-director border test): q_1 = k0 -
    // m0 t.  All P directors at once with GSUM would spill (slower).
    constexpr bool SYM = BORDER == 2;
    constexpr int NP = GSUM && !SYM ? 2 : P;
    static_assert(P % NP == 0 && (!GSUM || PP <= 2), "director split");
#pragma unroll 1
    for (int half = 0; half < P / NP; ++half) {
        AdjAcc a2[NP];
        adj_zero(a2);
        double ux[NP], uy[NP], uz[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int o = min(obase + G * (NP * half + p), y.O - 1);
            ux[p] = y.axes[3 * o];
            uy[p] = y.axes[3 * o + 1];
            uz[p] = y.axes[3 * o + 2];
        }
        const NearGeom g = near_geom(cx, cy, cz, y.off0, y.off1, y.rc2, y.floor_out2);
        ChunkPlan plan;
        plan.init_range(r.off, r.n_near, r.n_near);
        stage_prologue(st, plan, y.hi, y.lo, seq);
        double sh_half = 0.0;
        for (int c = 0; c < plan.n_chunks; ++c) {
            if (!stage_wait(st, plan, c, seq, a.status)) return false;
            int start, len;
            bool near;
            plan.chunk(c, start, len, near);
            const int s = (seq + c) % kStages;
            near_convert<NT>(st.hib + s * kCH, st.lob + s * kCH, ed, len);
            __syncthreads();
            if (y.near_mode == 2)
                near_chunk_adj<NP, 2, SYM>(ed, std4, len, g, ux, uy, uz, a2, sh_half);
            else
                near_chunk_adj<NP, 1, SYM>(ed, std4, len, g, ux, uy, uz, a2, sh_half);
            stage_next(st, plan, y.hi, y.lo, c, seq);
        }
        seq += plan.n_chunks;
        if (half == 0) shift_sum = sh_half;   // the same entries in every pass
        // acc indices stay compile-time constants (a runtime index would put
        // acc in local memory)
        if constexpr (GSUM) {
            grad_store<NT, NP, SYM>(gsum, a2, NP * half);
#pragma unroll
            for (int h = 0; h < P / NP; ++h)
                if (h == half)
#pragma unroll
                    for (int p = 0; p < NP; ++p) acc[NP * h + p].e = a2[p].e;
        } else {
#pragma unroll
            for (int p = 0; p < NP; ++p) acc[p] = a2[p];
        }
    }
    {
        float2 ux[PP], uy[PP], uz[PP];
#pragma unroll
        for (int j = 0; j < PP; ++j) {
            const int o0 = min(obase + G * (2 * j), y.O - 1);
            const int o1 = min(obase + G * (2 * j + 1), y.O - 1);
            ux[j] = make_float2((float)y.axes[3 * o0], (float)y.axes[3 * o1]);
            uy[j] = make_float2((float)y.axes[3 * o0 + 1], (float)y.axes[3 * o1 + 1]);
            uz[j] = make_float2((float)y.axes[3 * o0 + 2], (float)y.axes[3 * o1 + 2]);
        }
        const FarGeom g = far_geom(cx, cy, cz, y.off0, y.off1, y.rc2f);
        // inner entries, the shell, then (symmetric sites) the outer shell,
        // where only the near site of each director can be inside
        const int n_outer = SYM && OUTER ? r.n_outer : 0;
#pragma unroll 1
        for (int pass = 0; pass < 3; ++pass) {
            ChunkPlan plan;
            if (pass == 0)
                plan.init_range(r.off + r.n_near, 0, r.n_inner);
            else if (pass == 1)
                plan.init_range(r.off + r.n_near + r.n_inner, 0,
                                r.n_total - r.n_near - r.n_inner - n_outer);
            else
                plan.init_range(r.off + r.n_total - n_outer, 0, n_outer);
            stage_prologue(st, plan, y.hi, y.lo, seq);
            for (int c = 0; c < plan.n_chunks; ++c) {
                if (!stage_wait(st, plan, c, seq, a.status)) return false;
                int start, len;
                bool near;
                plan.chunk(c, start, len, near);
                const float4 *hb = st.hib + ((seq + c) % kStages) * kCH;
                constexpr int GNT = GSUM ? NT : 0;
                if (pass == 2) {
                    if constexpr (SYM && OUTER)
                        far_chunk_outer<P, FLUSH, UNROLL, GNT, BORDER>(hb, stf, len, g, ux, uy,
                                                                       uz, acc, gsum, border);
                } else if (pass == 1) {
                    far_chunk_adj<P, NEWTON, FLUSH, true, RCP1, UNROLL, GNT, BORDER, SYM>(
                        hb, stf, len, g, ux, uy, uz, acc, shift_sum, gsum, border);
                } else {
                    far_chunk_adj<P, NEWTON, FLUSH, false, RCP1, UNROLL, GNT, 0, SYM>(
                        hb, stf, len, g, ux, uy, uz, acc, shift_sum, gsum);
                }
                stage_next(st, plan, y.hi, y.lo, c, seq);
            }
            seq += plan.n_chunks;
        }
    }
    if constexpr (GSUM) grad_load<NT, P, SYM>(gsum, acc);
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int o = min(obase + G * p, y.O - 1);
        acc[p].e += 2.0 * shift_sum;
        adj_finish(acc[p], y.off0, y.off1, y.axes[3 * o], y.axes[3 * o + 1], y.axes[3 * o + 2],
                   e[p], gr[p]);
    }
    return true;
}

// ADJ: 0 = forward; forward + adjoint with the far reciprocal taken as
// 1 = rcp(q) cubed (default), 2 = rcp(q^3) + Newton, 3 = rcp(q^3);
// 5 = as 1 with the far entry loop unrolled twice; 6 / 7 = as 1 with the
// FP32 gradient partials flushed every 16 / 64 entries instead of once per
// 128-entry chunk; 8 = as 1 with the FP64 gradient sums in shared memory
// during the far passes (fewer registers: more resident CTAs); 11 / 12 = as
// 8 / 1 with the far entry loop unrolled twice; 17 = as 8 unrolled four
// times.  OUTER (symmetric sites, BORDER 2): the outer shell entries in the
// single-site pass (far_chunk_outer).  BORDER: 0 none, 1 the
// cutoff-border test per site (|q - rc^2|), 2 per director (| |d0 . u| -
// |T*| |, symmetric sites only).
template <int CB, int G, int P, int MINB, int ADJ, int BORDER = 0, bool OUTER = false>
__global__ void __launch_bounds__(CB *G, MINB) batch_field_kernel(BatchArgs a) {
    constexpr int NT = CB * G, PP = P / 2;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_item;
    Stager st;
    st.bar = reinterpret_cast<uint64_t *>(smem);
    st.hib = reinterpret_cast<float4 *>(smem + 64);
    st.lob = st.hib + kStages * kCH;
    double *ed = reinterpret_cast<double *>(st.lob + kStages * kCH);   // [kCH][4]
    float4 *stf = reinterpret_cast<float4 *>(ed + 4 * kCH);
    const int tid = threadIdx.x;
    constexpr bool kGsum = ADJ == 8 || ADJ == 11 || ADJ == 17;
    constexpr int kUnroll = ADJ == 17 ? 4 : ADJ == 5 || ADJ == 11 || ADJ == 12 ? 2 : 1;
    init_barriers(st);
    int last_sys = -1;
    unsigned seq = 0;
    while (true) {
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= a.n_items) break;
        const int4 w = a.items[it];
        const BatchSys &y = a.sys[w.x];
        double *std4 = reinterpret_cast<double *>(stf + y.n_types);
        if (w.x != last_sys) {
            load_types<NT>(stf, std4, y.tf, y.td, y.n_types);
            last_sys = w.x;
        }
        __syncthreads();
        const RegionInfo r = y.regs[w.y];
        const int cl = tid % CB, og = tid / CB;
        const bool cvalid = cl < r.ni * r.nj * r.nk;
        const int clc = cvalid ? cl : 0;
        const int gk = r.k0 + clc % r.nk, gj = r.j0 + (clc / r.nk) % r.nj,
                  gi = r.i0 + clc / (r.nk * r.nj);
        double cx, cy, cz;
        frac_to_cart(y.H, (gi + .5) / y.S - r.of[0], (gj + .5) / y.S - r.of[1],
                     (gk + .5) / y.S - r.of[2], cx, cy, cz);
        const int obase = w.z * (G * P) + og;
        double e[P];
        double gr[ADJ ? P : 1][6];
        float border[ADJ ? P : 1];
        if constexpr (ADJ) {
            double *gsum = reinterpret_cast<double *>(std4 + 4 * y.n_types);
            if (!batch_item_adj<CB, G, P, ADJ == 2, ADJ == 1 || ADJ >= 5, kUnroll,
                                ADJ == 6 ? 16 : ADJ == 7 ? 64 : 128, kGsum, BORDER, OUTER>(
                    a, y, r, st, ed, stf, std4, gsum, seq, cx, cy, cz, obase, e, gr, border))
                return;
        } else {
        // ---- near pairs (FP64)
        {
            double ux[P], uy[P], uz[P], acc[P][2];
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const int o = min(obase + G * p, y.O - 1);
                ux[p] = y.axes[3 * o];
                uy[p] = y.axes[3 * o + 1];
                uz[p] = y.axes[3 * o + 2];
                acc[p][0] = acc[p][1] = 0.0;
            }
            const NearGeom g = near_geom(cx, cy, cz, y.off0, y.off1, y.rc2, y.floor_out2);
            double shift_near = 0.0;
            ChunkPlan plan;
            plan.init_range(r.off, r.n_near, r.n_near);
            stage_prologue(st, plan, y.hi, y.lo, seq);
            for (int c = 0; c < plan.n_chunks; ++c) {
                if (!stage_wait(st, plan, c, seq, a.status)) return;
                int start, len;
                bool near;
                plan.chunk(c, start, len, near);
                const int s = (seq + c) % kStages;
                near_convert<NT>(st.hib + s * kCH, st.lob + s * kCH, ed, len);
                __syncthreads();
                if (y.near_mode == 2)
                    near_chunk<P, 2>(ed, std4, len, g, ux, uy, uz, acc, shift_near);
                else
                    near_chunk<P, 1>(ed, std4, len, g, ux, uy, uz, acc, shift_near);
                stage_next(st, plan, y.hi, y.lo, c, seq);
            }
            seq += plan.n_chunks;
#pragma unroll
            for (int p = 0; p < P; ++p) e[p] = acc[p][0] + acc[p][1] + 2.0 * shift_near;
        }
        // ---- far pairs (packed FP32x2)
        {
            float2 ux[PP], uy[PP], uz[PP];
            double acc[P];
#pragma unroll
            for (int j = 0; j < PP; ++j) {
                const int o0 = min(obase + G * (2 * j), y.O - 1);
                const int o1 = min(obase + G * (2 * j + 1), y.O - 1);
                ux[j] = make_float2((float)y.axes[3 * o0], (float)y.axes[3 * o1]);
                uy[j] = make_float2((float)y.axes[3 * o0 + 1], (float)y.axes[3 * o1 + 1]);
                uz[j] = make_float2((float)y.axes[3 * o0 + 2], (float)y.axes[3 * o1 + 2]);
                acc[2 * j] = acc[2 * j + 1] = 0.0;
            }
            const FarGeom g = far_geom(cx, cy, cz, y.off0, y.off1, y.rc2f);
            double shift_sum = 0.0;
            // inner entries, then the shell, whose outer entries (symmetric
            // sites) take the near site of each director alone
            const int shell_n = r.n_total - r.n_near - r.n_inner;
            const bool sym = y.off0 != 0.0 && y.off1 == -y.off0;
            const int outer_at = shell_n - (sym ? r.n_outer : 0);
#pragma unroll 1
            for (int pass = 0; pass < 2; ++pass) {
                ChunkPlan plan;
                plan.init_range(r.off + r.n_near + (pass ? r.n_inner : 0), 0,
                                pass ? shell_n : r.n_inner);
                stage_prologue(st, plan, y.hi, y.lo, seq);
                for (int c = 0; c < plan.n_chunks; ++c) {
                    if (!stage_wait(st, plan, c, seq, a.status)) return;
                    int start, len;
                    bool near;
                    plan.chunk(c, start, len, near);
                    const float4 *hb = st.hib + ((seq + c) % kStages) * kCH;
                    if (pass && sym)
                        far_chunk_fwd<P, 16, true, true>(hb, stf, len, g, ux, uy, uz, acc,
                                                         shift_sum, outer_at - start);
                    else if (pass)
                        far_chunk_fwd<P, 16, true>(hb, stf, len, g, ux, uy, uz, acc, shift_sum);
                    else
                        far_chunk_fwd<P, 16, false>(hb, stf, len, g, ux, uy, uz, acc, shift_sum);
                    stage_next(st, plan, y.hi, y.lo, c, seq);
                }
                seq += plan.n_chunks;
            }
#pragma unroll
            for (int p = 0; p < P; ++p) e[p] += acc[p] + 2.0 * shift_sum;
        }
        }
        if (cvalid) {
            const long long S3 = (long long)y.S * y.S * y.S;
            const long long cg = ((long long)gi * y.S + gj) * y.S + gk;
#pragma unroll
            for (int j = 0; j < PP; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int o = obase + G * (2 * j + h);
                    const double v = e[2 * j + h];
                    if (o < y.O) {
                        const long long idx = (long long)o * S3 + cg;
                        y.out[idx] = (float)v;
                        if (y.out64) y.out64[idx] = v;
                        if constexpr (ADJ) {
                            float2 *gd = reinterpret_cast<float2 *>(y.grad + 6 * idx);
                            const double *gp = gr[2 * j + h];
                            gd[0] = make_float2((float)gp[0], (float)gp[1]);
                            gd[1] = make_float2((float)gp[2], (float)gp[3]);
                            gd[2] = make_float2((float)gp[4], (float)gp[5]);
                        }
                        const bool band = v > a.band_lo && v < a.band_hi;
                        bool near_rc = false;
                        if constexpr (ADJ && BORDER) {
                            // |q - rc^2|, or its director-space estimate scaled by 2 |o|
                            near_rc = BORDER == 2 ? border[2 * j + h] * (float)(2.0 * fabs(y.off0)) <
                                                        kBorderTolDir
                                                  : border[2 * j + h] < kBorderTol;
                        }
                        if (band || near_rc) {
                            // band poses are re-evaluated in FP64, the others
                            // (kRepairOnly) only have their shell pairs re-tested
                            const int k = atomicAdd(&a.refine[0], 1);
                            if (k < a.refine_cap) {
                                a.refine[1 + 2 * k] =
                                    w.x | (band || a.full_refine ? 0 : kRepairOnly);
                                a.refine[2 + 2 * k] = (int)idx;
                            }
                        }
                    }
                }
        }
    }
}

// FP64 re-evaluation of the flagged poses, one warp per pose.
__global__ void batch_refine_kernel(BatchArgs a) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int count = min(a.refine[0], a.refine_cap);
    for (int q = warp; q < count; q += nwarps) {
        const BatchSys &y = a.sys[a.refine[1 + 2 * q]];
        const long long idx = a.refine[2 + 2 * q];
        const long long S3 = (long long)y.S * y.S * y.S;
        const int o = (int)(idx / S3);
        const long long c = idx % S3;
        const int gi = (int)(c / ((long long)y.S * y.S)), gj = (int)((c / y.S) % y.S),
                  gk = (int)(c % y.S);
        const RegionInfo r = y.regs[((gi / y.bi) * y.nrj + gj / y.bj) * y.nrk + gk / y.bk];
        double cx, cy, cz;
        frac_to_cart(y.H, (gi + .5) / y.S - r.of[0], (gj + .5) / y.S - r.of[1],
                     (gk + .5) / y.S - r.of[2], cx, cy, cz);
        const double ux = y.axes[3 * o], uy = y.axes[3 * o + 1], uz = y.axes[3 * o + 2];
        double sum = 0.0;
        for (int s = 0; s < 2; ++s) {
            const double off = s ? y.off1 : y.off0;
            const double px = cx + off * ux, py = cy + off * uy, pz = cz + off * uz;
            for (int k = lane; k < r.n_total; k += 32) {
                const float4 h = y.hi[r.off + k], l = y.lo[r.off + k];
                const double dx = px - ((double)h.x + (double)l.x);
                const double dy = py - ((double)h.y + (double)l.y);
                const double dz = pz - ((double)h.z + (double)l.z);
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 >= y.rc2) continue;
                const int t = __float_as_int(h.w);
                const double fl = y.td[4 * t + 3];
                const double s2 = d2 < fl ? fl : d2;
                const double i2 = 1.0 / s2;
                const double i6 = i2 * i2 * i2;
                sum += y.td[4 * t] * i6 * i6 - y.td[4 * t + 1] * i6 + y.td[4 * t + 2];
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
        if (lane == 0) {
            y.out[idx] = (float)sum;
            if (y.out64) y.out64[idx] = sum;
        }
    }
}

// FP64 re-evaluation of the flagged poses of a forward + adjoint batch, one
// warp per pose, the lanes striding over the region's list:
// * poses in the refinement band: energy and gradient from every pair in
//   FP64 (fp64_pose_pairs_both, the pair test and terms of
//   plain_fp64_adj_kernel);
// * poses with a shell pair within kBorderTol of the cutoff (kRepairOnly):
//   each shell pair's inside/outside decision is recomputed with the far
//   kernel's own FP32 arithmetic (bit for bit: the same operations in the
//   same order, so the same roundings) and with the FP64 test the oracle
//   uses (d2 >= rc^2 out); where they differ, the pair's FP64 energy and
//   gradient terms are added (FP64 inside) or removed (FP64 outside).  Every
//   other pair of the pose was already decided the same way by both.
__global__ void batch_refine_adj_kernel(BatchArgs a) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int count = min(a.refine[0], a.refine_cap);
    for (int q = warp; q < count; q += nwarps) {
        const int tag = a.refine[1 + 2 * q];
        const bool repair = (tag & kRepairOnly) != 0;
        const BatchSys &y = a.sys[tag & ~kRepairOnly];
        const long long idx = a.refine[2 + 2 * q];
        const long long S3 = (long long)y.S * y.S * y.S;
        const int o = (int)(idx / S3);
        const long long c = idx % S3;
        const int gi = (int)(c / ((long long)y.S * y.S)), gj = (int)((c / y.S) % y.S),
                  gk = (int)(c % y.S);
        const RegionInfo r = y.regs[((gi / y.bi) * y.nrj + gj / y.bj) * y.nrk + gk / y.bk];
        double cx, cy, cz;
        frac_to_cart(y.H, (gi + .5) / y.S - r.of[0], (gj + .5) / y.S - r.of[1],
                     (gk + .5) / y.S - r.of[2], cx, cy, cz);
        const double u[3] = {y.axes[3 * o], y.axes[3 * o + 1], y.axes[3 * o + 2]};
        double e = 0.0, g[6];
        if (repair)
            shell_border_repair(y.hi, y.lo, y.td, r.off + r.n_near + r.n_inner,
                                r.n_total - r.n_near - r.n_inner, lane, 32, y.rc2, y.rc2f,
                                y.off0, y.off1, cx, cy, cz, u, e, g);
        else
            fp64_pose_pairs_both(y.hi, y.lo, y.td, r.off, r.n_total, lane, 32, y.rc2, y.off0,
                                 y.off1, cx, cy, cz, u, e, g);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, off);
#pragma unroll
            for (int k = 0; k < 6; ++k) g[k] += __shfl_xor_sync(0xffffffffu, g[k], off);
        }
        if (lane == 0) {
            fp64_tangent(u, g);
            float2 *gd = reinterpret_cast<float2 *>(y.grad + 6 * idx);
            if (repair) {
                // corrections on top of the far kernel's results
                const double e64 = (y.out64 ? y.out64[idx] : (double)y.out[idx]) + e;
                y.out[idx] = (float)e64;
                if (y.out64) y.out64[idx] = e64;
                const float2 g0 = gd[0], g1 = gd[1], g2 = gd[2];
                gd[0] = make_float2((float)((double)g0.x + g[0]), (float)((double)g0.y + g[1]));
                gd[1] = make_float2((float)((double)g1.x + g[2]), (float)((double)g1.y + g[3]));
                gd[2] = make_float2((float)((double)g2.x + g[4]), (float)((double)g2.y + g[5]));
            } else {
                y.out[idx] = (float)e;
                if (y.out64) y.out64[idx] = e;
                gd[0] = make_float2((float)g[0], (float)g[1]);
                gd[1] = make_float2((float)g[2], (float)g[3]);
                gd[2] = make_float2((float)g[4], (float)g[5]);
            }
        }
    }
}

// ---------------------------------------------------------------- host side

struct BatchConfig {
    int shape;   // index into the mode's kernel table (batch_kernel)
    int grid;    // resident CTAs (persistent grid)
};

// CTA shapes <CB centers, G director groups, P directors per thread> the
// autotuner chooses from; a table's shapes share CB and the director block
// G x P (16 x 32 or 8 x 64).  Forward: 128 threads x 4 directors or 256 x 2.
// Forward + adjoint (9 FP64 sums per director): 256 x 2, or 128 x 4 bounded
// to 2 or 3 CTAs per SM (225 / 168 registers), or 128 x 4 with the FP64
// gradient sums in shared memory (162 registers, 3 CTAs per SM).
struct BatchKernel {
    void (*fn)(BatchArgs);
    int threads;
    const char *name;
};

static const BatchKernel kForwardKernels[] = {
    {batch_field_kernel<16, 8, 4, 4, 0>, 128, "128x4"},
    {batch_field_kernel<16, 16, 2, 3, 0>, 256, "256x2"}};
static const BatchKernel kAdjointKernels[] = {
    {batch_field_kernel<16, 16, 2, 2, 1, true>, 256, "256x2"},
    {batch_field_kernel<16, 8, 4, 2, 1, true>, 128, "128x4"},
    {batch_field_kernel<16, 8, 4, 3, 1, true>, 128, "128x4/3"},
    {batch_field_kernel<16, 16, 2, 2, 5, true>, 256, "256x2 unroll2"},
    {batch_field_kernel<16, 8, 4, 3, 8, true>, 128, "128x4/3 gsum"}};
static const BatchKernel kAdjointNewtonKernels[] = {   // accuracy/speed study
    {batch_field_kernel<16, 16, 2, 2, 2>, 256, "256x2 rcp3+newton"},
    {batch_field_kernel<16, 8, 4, 2, 2>, 128, "128x4 rcp3+newton"}};
static const BatchKernel kAdjointRcp3Kernels[] = {     // accuracy/speed study
    {batch_field_kernel<16, 16, 2, 2, 3>, 256, "256x2 rcp3"},
    {batch_field_kernel<16, 8, 4, 2, 3>, 128, "128x4 rcp3"}};
static const BatchKernel kAdjointFlush16Kernels[] = {   // accuracy/speed study
    {batch_field_kernel<16, 16, 2, 2, 6>, 256, "256x2 flush16"},
    {batch_field_kernel<16, 8, 4, 2, 6>, 128, "128x4 flush16"}};
static const BatchKernel kAdjointFlush64Kernels[] = {   // accuracy/speed study
    {batch_field_kernel<16, 16, 2, 2, 7>, 256, "256x2 flush64"},
    {batch_field_kernel<16, 8, 4, 2, 7>, 128, "128x4 flush64"}};
// 8-center regions x 64-director items (the same 512 poses per staged
// entry): a smaller region radius, hence shorter near and shell lists
static const BatchKernel kForwardCb8Kernels[] = {
    {batch_field_kernel<8, 16, 4, 4, 0>, 128, "8c 128x4"},
    {batch_field_kernel<8, 32, 2, 3, 0>, 256, "8c 256x2"}};
// symmetric sites: border per director, outer shell in the single-site pass
static const BatchKernel kAdjointCb8Kernels[] = {
    {batch_field_kernel<8, 16, 4, 3, 8, 2, true>, 128, "8c 128x4/3 gsum"},
    {batch_field_kernel<8, 16, 4, 2, 1, 2, true>, 128, "8c 128x4"},
    {batch_field_kernel<8, 32, 2, 2, 1, 2, true>, 256, "8c 256x2"},
    {batch_field_kernel<8, 16, 4, 3, 11, 2, true>, 128, "8c 128x4/3 gsum unroll2"},
    {batch_field_kernel<8, 16, 4, 2, 12, 2, true>, 128, "8c 128x4 unroll2"},
    {batch_field_kernel<8, 16, 4, 3, 17, 2, true>, 128, "8c 128x4/3 gsum unroll4"}};
// the same with the outer shell in the two-site shell pass (timing study)
static const BatchKernel kAdjointCb8TwoSiteKernels[] = {
    {batch_field_kernel<8, 16, 4, 3, 11, 2>, 128, "8c 128x4/3 gsum unroll2, two-site outer"},
    {batch_field_kernel<8, 16, 4, 3, 17, 2>, 128, "8c 128x4/3 gsum unroll4, two-site outer"}};
static const BatchKernel kAdjointCb8SiteBorderKernels[] = {   // any sites: border per site
    {batch_field_kernel<8, 16, 4, 3, 8, 1>, 128, "8c 128x4/3 gsum, border/site"},
    {batch_field_kernel<8, 16, 4, 2, 1, 1>, 128, "8c 128x4, border/site"},
    {batch_field_kernel<8, 32, 2, 2, 1, 1>, 256, "8c 256x2, border/site"},
    {batch_field_kernel<8, 16, 4, 3, 11, 1>, 128, "8c 128x4/3 gsum unroll2, border/site"},
    {batch_field_kernel<8, 16, 4, 2, 12, 1>, 128, "8c 128x4 unroll2, border/site"},
    {batch_field_kernel<8, 16, 4, 3, 17, 1>, 128, "8c 128x4/3 gsum unroll4, border/site"}};
// the same without the cutoff-border test (timing study: its cost)
static const BatchKernel kAdjointCb8NoBorderKernels[] = {
    {batch_field_kernel<8, 16, 4, 3, 8>, 128, "8c 128x4/3 gsum, no border test"},
    {batch_field_kernel<8, 16, 4, 2, 1>, 128, "8c 128x4, no border test"},
    {batch_field_kernel<8, 32, 2, 2, 1>, 256, "8c 256x2, no border test"}};
constexpr int kMaxCandidates = 12;

#define VEXT_COUNT(t) (int)(sizeof t / sizeof t[0])

// kind: 0 forward, 1 forward + adjoint (reciprocal of q, cubed),
// 2 with the reciprocal of q^3 and a Newton step, 3 the same without it,
// 4 / 5 default with FP32 gradient partials over 16 / 64 entries (a whole
// 128-entry chunk by default; the energy partials always cover 16), 6 default
// on 8-center regions with 64-director items, 7 forward on 8-center regions,
// 8 as 6 without the cutoff-border test, 9 as 6 with the border test per site
// (guests whose sites are not symmetric about the center), 10 as 6 with the
// outer shell in the two-site shell pass
static int batch_kernel_count(int kind) {
    switch (kind) {
    case 0: return VEXT_COUNT(kForwardKernels);
    case 1: return VEXT_COUNT(kAdjointKernels);
    case 2: return VEXT_COUNT(kAdjointNewtonKernels);
    case 4: return VEXT_COUNT(kAdjointFlush16Kernels);
    case 5: return VEXT_COUNT(kAdjointFlush64Kernels);
    case 6: return VEXT_COUNT(kAdjointCb8Kernels);
    case 7: return VEXT_COUNT(kForwardCb8Kernels);
    case 8: return VEXT_COUNT(kAdjointCb8NoBorderKernels);
    case 9: return VEXT_COUNT(kAdjointCb8SiteBorderKernels);
    case 10: return VEXT_COUNT(kAdjointCb8TwoSiteKernels);
    default: return VEXT_COUNT(kAdjointRcp3Kernels);
    }
}

static const BatchKernel &batch_kernel(int kind, int shape) {
    switch (kind) {
    case 0: return kForwardKernels[shape];
    case 1: return kAdjointKernels[shape];
    case 2: return kAdjointNewtonKernels[shape];
    case 4: return kAdjointFlush16Kernels[shape];
    case 5: return kAdjointFlush64Kernels[shape];
    case 6: return kAdjointCb8Kernels[shape];
    case 7: return kForwardCb8Kernels[shape];
    case 8: return kAdjointCb8NoBorderKernels[shape];
    case 9: return kAdjointCb8SiteBorderKernels[shape];
    case 10: return kAdjointCb8TwoSiteKernels[shape];
    default: return kAdjointRcp3Kernels[shape];
    }
}

// The kernel table of a batch: forward on 16-center regions (0,
// centers_per_region 16 or 32) or, by default, on 8-center regions (7); the
// forward + adjoint studies (2-5, selected by variant bits), forward +
// adjoint on 16-center regions (1) or, by default, on 8-center regions (6).
static int batch_kind(const Options &o, bool adj) {
    const bool cb16 = o.cb == 16 || o.cb == 32;
    if (!adj) return cb16 ? 0 : 7;
    if (o.variant & 32) return 2;
    if (o.variant & 64) return 3;
    if (o.variant & 128) return 4;
    if (o.variant & 512) return 5;
    if (o.variant & 1024) return cb16 ? 1 : 8;
    if (o.variant & 8192) return cb16 ? 1 : 10;
    return cb16 ? 1 : 6;
}

int batch_item_directors(const Options &o, bool adj) {
    const int kind = batch_kind(o, adj);
    return kind >= 6 && kind <= 10 ? 64 : 32;
}

}  // namespace vext

using namespace vext;

struct vext_batch_s {
    std::vector<vext_system> systems;
    int size = 0, n_axes = 0;
    Options opt;
    BatchSys *d_sys = nullptr;
    std::vector<std::pair<float *, float *>> targets;   // current (out, grad) of each system
    int4 *d_items = nullptr, *d_sample = nullptr;
    int n_items = 0, n_sample = 0;
    int *d_counter = nullptr, *d_refine = nullptr;
    int refine_cap = 0;
    double *d_axes = nullptr;
    int *d_status = nullptr;
    int max_types = 0;
    int64_t poses = 0, list_bytes = 0;
    BatchConfig config{0, 0};
    bool adj = false;
    int kind = 0;   // batch_kernel table
    BatchConfig cands[kMaxCandidates] = {};
    int n_cands = 0;
    float tune_ms[kMaxCandidates] = {};
    bool tune_cached = false;   // the pick came from the process-wide tuning cache
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~vext_batch_s() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaFree(d_sys);
        cudaFree(d_items);
        cudaFree(d_sample);
        cudaFree(d_counter);
        cudaFree(d_refine);
        cudaFree(d_axes);
        cudaFree(d_status);
        if (stream) cudaStreamDestroy(stream);
    }
};

// Staging + converted near chunk + type tables (+ the FP64 gradient sums of
// 16 centers x 32 directors for the adjoint kernels that park them there).
static size_t batch_smem(int max_types, bool adj) {
    return kStageBytes + (size_t)kCH * 4 * sizeof(double) + (size_t)max_types * 48 +
           (adj ? (size_t)kGradWords * 16 * 32 * sizeof(double) : 0);
}

static int batch_launch(vext_batch b, const BatchConfig &cfg, const int4 *items, int n_items,
                        cudaStream_t st) {
    BatchArgs a;
    a.sys = b->d_sys;
    a.items = items;
    a.n_items = n_items;
    a.counter = b->d_counter;
    a.refine = b->d_refine;
    a.refine_cap = b->refine_cap;
    a.band_lo = b->opt.band_lo;
    a.band_hi = b->opt.band_hi;
    a.full_refine = (b->opt.variant & kVariantFullRefine) != 0;
    a.status = b->d_status;
    const size_t smem = batch_smem(b->max_types, b->adj);
    VEXT_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(int), st));
    VEXT_CUDA(cudaMemsetAsync(b->d_refine, 0, sizeof(int), st));
    const BatchKernel &k = batch_kernel(b->kind, cfg.shape);
    k.fn<<<cfg.grid, k.threads, smem, st>>>(a);
    VEXT_CUDA(cudaGetLastError());
    if (b->adj) {
        batch_refine_adj_kernel<<<1184, 256, 0, st>>>(a);
        VEXT_CUDA(cudaGetLastError());
    } else if (b->opt.band_hi > b->opt.band_lo) {
        batch_refine_kernel<<<1184, 256, 0, st>>>(a);
        VEXT_CUDA(cudaGetLastError());
    }
    return 0;
}

namespace vext {

// Autotuner picks per (device, kernel table, size class).
struct TuneKey {
    int dev, kind, size_class;
    bool operator<(const TuneKey &o) const {
        return std::tie(dev, kind, size_class) < std::tie(o.dev, o.kind, o.size_class);
    }
};
struct TunePick {
    int shape, grid;
    float ms[kMaxCandidates];
};
static std::mutex g_tune_lock;
static std::map<TuneKey, TunePick> g_tune_cache;
// vext_options.variant bit: time the candidates even when the cache holds a
// pick for this class (the pick is then replaced)
constexpr int kVariantTuneAfresh = 2048;

// Shared by vext_batch_create, vext_batch_create_adjoint and the cached
// one-system batch of vext_field_adjoint_device (which already holds its
// system's lock: lock_systems = false).
int batch_build(int n_systems, const vext_system *systems, int size, int n_axes,
                const double *axes, const vext_options *opt, float *const *outputs,
                float *const *gradients, double *const *outputs_f64, bool lock_systems,
                vext_batch *out) {
    if (!out || n_systems < 1 || !systems || !outputs || size < 1 || n_axes < 1 || !axes)
        return fail(VEXT_ERR_ARGUMENT, "bad batch arguments");
    for (int k = 0; k < n_systems; ++k)
        if (!systems[k] || !outputs[k] || (gradients && !gradients[k]))
            return fail(VEXT_ERR_ARGUMENT, "null system or output %d", k);
    *out = nullptr;
    const long long S3 = (long long)size * size * size;
    if (S3 * n_axes >= (1LL << 31) - 1)
        return fail(VEXT_ERR_CAPACITY, "size^3 * n_axes must stay below 2^31");
    for (int k = 0; k < 3 * n_axes; ++k)
        if (!std::isfinite(axes[k])) return fail(VEXT_ERR_ARGUMENT, "non-finite director");
    auto *b = new vext_batch_s();
    std::unique_ptr<vext_batch_s> guard(b);
    b->systems.assign(systems, systems + n_systems);
    b->size = size;
    b->n_axes = n_axes;
    b->opt = resolve_options(opt);
    b->adj = gradients != nullptr;
    b->kind = batch_kind(b->opt, b->adj);
    if (b->opt.mode != VEXT_MODE_MIXED)
        return fail(VEXT_ERR_ARGUMENT, "batched fields run in the mixed mode only");
    int dev = 0;
    VEXT_CUDA(cudaGetDevice(&dev));
    VEXT_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    VEXT_CUDA(cudaMalloc(&b->d_axes, sizeof(double) * 3 * n_axes));
    VEXT_CUDA(cudaMemcpy(b->d_axes, axes, sizeof(double) * 3 * n_axes, cudaMemcpyHostToDevice));
    // regions of 16 centers x items of 32 directors, or 8 x 64 (kinds 6-9)
    const int kOB = batch_item_directors(b->opt, b->adj), cb = 512 / kOB;
    std::vector<BatchSys> hs(n_systems);
    std::vector<std::pair<long long, int4>> items;
    // Systems with the same framework (equal frame_hash; in the benchmark's
    // batches, one framework with two guests) share one region-list set,
    // built by the member with the largest site offset: its lists hold every
    // image the others need (a larger list radius, a near list that covers
    // theirs, an inner class inside theirs), and each member keeps its own
    // offsets and type table.
    std::vector<int> owner(n_systems);
    for (int k = 0; k < n_systems; ++k) {
        owner[k] = k;
        for (int j = 0; j < k; ++j) {
            const System &a = systems[j]->sys, &c = systems[k]->sys;
            if (owner[j] == j && a.frame_hash == c.frame_hash && a.device == c.device) {
                owner[k] = j;
                if (c.max_offset > systems[owner[k]]->sys.max_offset) {
                    for (int i = 0; i < k; ++i)
                        if (owner[i] == j) owner[i] = k;
                    owner[k] = k;
                }
                break;
            }
        }
    }
    std::vector<RegionSet *> lists(n_systems, nullptr);
    for (int k = 0; k < n_systems; ++k) {
        if (owner[k] != k) continue;
        System *sys = &systems[k]->sys;
        if (sys->device != dev)
            return fail(VEXT_ERR_ARGUMENT, "system %d lives on another device", k);
        std::unique_lock<std::mutex> lock(sys->lock, std::defer_lock);
        if (lock_systems) lock.lock();
        VEXT_TRY(get_field_regions(sys, size, cb, b->opt.r_split, &lists[k], sys->stream));
        b->list_bytes += lists[k]->n_entries * 32;
    }
    {
        size_t n = 0;
        for (int k = 0; k < n_systems; ++k)
            n += (size_t)lists[owner[k]]->n_regions * ((n_axes + kOB - 1) / kOB);
        items.reserve(n);
    }
    for (int k = 0; k < n_systems; ++k) {
        System *sys = &systems[k]->sys;
        if (sys->device != dev)
            return fail(VEXT_ERR_ARGUMENT, "system %d lives on another device", k);
        const System *list_sys = &systems[owner[k]]->sys;
        RegionSet *rs = lists[owner[k]];
        BatchSys &y = hs[k];
        y.H = sys->H;
        y.rc2 = sys->cutoff * sys->cutoff;
        y.rc2f = (float)y.rc2;
        y.off0 = sys->offsets[0];
        y.off1 = sys->offsets[1];
        y.floor_out2 = floor_clear_radius2(*sys);
        y.S = size;
        y.O = n_axes;
        y.axes = b->d_axes;
        y.regs = rs->d_info;
        y.hi = rs->d_hi;
        y.lo = rs->d_lo;
        y.tf = sys->d_tf;
        y.td = sys->d_td;
        y.n_types = sys->n_types;
        double rho = 0;
        for (const RegionInfo &r : rs->h_info) rho = std::max(rho, r.rho);
        y.near_mode =
            rs->r_split + 2.0 * (rho + list_sys->max_offset) + 1e-6 < sys->cutoff ? 2 : 1;
        y.bi = rs->bi;
        y.bj = rs->bj;
        y.bk = rs->bk;
        y.nrj = rs->n_rj;
        y.nrk = rs->n_rk;
        y.out = outputs[k];
        y.grad = gradients ? gradients[k] : nullptr;
        y.out64 = outputs_f64 ? outputs_f64[k] : nullptr;
        b->max_types = std::max(b->max_types, sys->n_types);
        b->poses += S3 * n_axes;
        const int n_ob = (n_axes + kOB - 1) / kOB;
        for (int ri = 0; ri < rs->n_regions; ++ri)
            for (int ob = 0; ob < n_ob; ++ob)
                items.push_back({(long long)rs->h_info[ri].n_total, make_int4(k, ri, ob, 0)});
    }
    // longest items first: a counting sort on the list length (stable, O(n);
    // the 100-field batches hold 2.7 M items)
    long long max_len = 0;
    for (const auto &it : items) max_len = std::max(max_len, it.first);
    std::vector<int64_t> start((size_t)max_len + 2, 0);
    for (const auto &it : items) ++start[(size_t)(max_len - it.first) + 1];
    for (size_t l = 1; l < start.size(); ++l) start[l] += start[l - 1];
    std::vector<int4> hitems(items.size());
    for (const auto &it : items) hitems[(size_t)start[(size_t)(max_len - it.first)]++] = it.second;
    b->n_items = (int)hitems.size();
    // the tuning sample: a strided subset of the queue (so it keeps the mix of
    // long and short items), every 128th item for large queues but at least
    // 16 items per SM, so that the persistent CTAs stay busy while it is
    // timed; each candidate is timed twice and keeps its better time
    int sms = 0;
    VEXT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t n_all = hitems.size();
    const size_t stride =
        std::max<size_t>(1, std::min<size_t>(128, n_all / std::max<size_t>(1, (size_t)sms * 16)));
    std::vector<int4> sample;
    for (size_t i = 0; i < n_all; i += stride) sample.push_back(hitems[i]);
    b->n_sample = (int)sample.size();
    // size class for the tuning cache: rounded log2 of the mean list length
    // per item and of the item count
    double mean_len = 0;
    for (const auto &it : items) mean_len += (double)it.first;
    mean_len /= (double)std::max<size_t>(items.size(), 1);
    const int size_class =
        (int)std::lround(std::log2(std::max(mean_len, 1.0))) * 64 +
        (int)std::lround(std::log2((double)std::max<size_t>(items.size(), 1)));
    // kinds 6 and 10 (the per-director border test, q_1 from the site-0
    // terms, the single-site outer shell pass of kind 6) assume exactly
    // symmetric sites, o_1 = -o_0 != 0 (two identical sites
    // about their center of mass); other guests take the same shapes with the
    // per-site test and both sites' terms
    if (b->kind == 6 || b->kind == 10)
        for (const BatchSys &y : hs)
            if (y.off0 == 0.0 || y.off1 != -y.off0) b->kind = 9;
    for (const BatchSys &y : hs) b->targets.push_back({y.out, y.grad});
    VEXT_CUDA(cudaMalloc(&b->d_sys, sizeof(BatchSys) * n_systems));
    VEXT_CUDA(cudaMemcpy(b->d_sys, hs.data(), sizeof(BatchSys) * n_systems, cudaMemcpyHostToDevice));
    VEXT_CUDA(cudaMalloc(&b->d_items, sizeof(int4) * hitems.size()));
    VEXT_CUDA(cudaMemcpy(b->d_items, hitems.data(), sizeof(int4) * hitems.size(),
                         cudaMemcpyHostToDevice));
    VEXT_CUDA(cudaMalloc(&b->d_sample, sizeof(int4) * sample.size()));
    VEXT_CUDA(cudaMemcpy(b->d_sample, sample.data(), sizeof(int4) * sample.size(),
                         cudaMemcpyHostToDevice));
    VEXT_CUDA(cudaMalloc(&b->d_counter, sizeof(int)));
    // refinement records (2 ints each): one pose in 8 at most, 512 MB at most
    // (the 100-field benchmark batch flags 0.75 % of its poses)
    b->refine_cap = (int)std::min<long long>(b->poses / 8 + 1024, 64LL << 20);
    VEXT_CUDA(cudaMalloc(&b->d_refine, sizeof(int) * (1 + 2 * (size_t)b->refine_cap)));
    VEXT_CUDA(cudaMalloc(&b->d_status, sizeof(int)));
    VEXT_CUDA(cudaMemset(b->d_status, 0, sizeof(int)));
    // ---- autotune: CTA shape x resident CTAs per SM, on the sampled queue
    const size_t smem = batch_smem(b->max_types, b->adj);
    // candidates: every kernel of the mode at its full occupancy, and at half
    // of it where that still leaves two or more CTAs per SM
    BatchConfig cands[kMaxCandidates];
    int n_cands = 0;
    const int n_kernels = batch_kernel_count(b->kind);
    if (b->opt.batch_shape < 0 || b->opt.batch_shape > n_kernels)
        return fail(VEXT_ERR_ARGUMENT, "batch_shape %d outside 0..%d", b->opt.batch_shape,
                    n_kernels);
    for (int k = 0; k < n_kernels; ++k) {
        if (b->opt.batch_shape && k != b->opt.batch_shape - 1) continue;   // pinned shape
        const BatchKernel &bk = batch_kernel(b->kind, k);
        VEXT_CUDA(cudaFuncSetAttribute(bk.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
        int occ = 0;
        VEXT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bk.fn, bk.threads, smem));
        if (occ < 1) continue;
        if (n_cands < kMaxCandidates) cands[n_cands++] = {k, sms * occ};
        if (occ >= 4 && n_cands < kMaxCandidates && !b->opt.batch_shape)
            cands[n_cands++] = {k, sms * (occ / 2)};
    }
    if (n_cands == 0) return fail(VEXT_ERR_CAPACITY, "batch kernel does not fit an SM");
    b->n_cands = n_cands;
    for (int c = 0; c < n_cands; ++c) b->cands[c] = cands[c];
    // a process-wide cache of the winners per (device, kernel table, size
    // class): later batches of the same class skip the timing runs
    const TuneKey key{dev, b->kind, size_class};
    bool cached = false;
    if (!b->opt.batch_shape && !(b->opt.variant & kVariantTuneAfresh)) {
        std::lock_guard<std::mutex> guard(g_tune_lock);
        auto hit = g_tune_cache.find(key);
        if (hit != g_tune_cache.end()) {
            for (int c = 0; c < n_cands; ++c)
                if (cands[c].shape == hit->second.shape && cands[c].grid == hit->second.grid) {
                    b->config = cands[c];
                    std::copy(hit->second.ms, hit->second.ms + kMaxCandidates, b->tune_ms);
                    cached = true;
                }
        }
    }
    if (!cached) {
        cudaEvent_t e0, e1;
        VEXT_CUDA(cudaEventCreate(&e0));
        VEXT_CUDA(cudaEventCreate(&e1));
        float best = 1e30f;
        const int n_warm = std::min(b->n_sample, sms);
        for (int c = 0; c < n_cands; ++c) {
            // warm-up on a few items (module load, first-launch costs)
            VEXT_TRY(batch_launch(b, cands[c], b->d_sample, n_warm, b->stream));
            float ms = 1e30f;
            for (int rep = 0; rep < 2; ++rep) {   // best of two: launch noise
                VEXT_CUDA(cudaEventRecord(e0, b->stream));
                VEXT_TRY(batch_launch(b, cands[c], b->d_sample, b->n_sample, b->stream));
                VEXT_CUDA(cudaEventRecord(e1, b->stream));
                VEXT_CUDA(cudaEventSynchronize(e1));
                float t = 0;
                VEXT_CUDA(cudaEventElapsedTime(&t, e0, e1));
                ms = std::min(ms, t);
            }
            b->tune_ms[c] = ms;
            if (ms < best) {
                best = ms;
                b->config = cands[c];
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (!b->opt.batch_shape) {
            std::lock_guard<std::mutex> guard(g_tune_lock);
            TunePick pick{b->config.shape, b->config.grid, {}};
            std::copy(b->tune_ms, b->tune_ms + kMaxCandidates, pick.ms);
            g_tune_cache[key] = pick;
        }
    }
    b->tune_cached = cached;
    int status = 0;
    VEXT_CUDA(cudaMemcpy(&status, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) return fail(VEXT_ERR_TIMEOUT, "a device wait gave up during batch tuning");
    // ---- capture the whole batch into a graph
    VEXT_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_launch(b, b->config, b->d_items, b->n_items, b->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    VEXT_CUDA(end);
    b->graph = g;
    VEXT_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    *out = guard.release();
    return 0;
}

}  // namespace vext

extern "C" int vext_batch_create(int n_systems, const vext_system *systems, int size,
                                 int n_axes, const double *axes, const vext_options *opt,
                                 float *const *outputs, vext_batch *out) {
    return batch_build(n_systems, systems, size, n_axes, axes, opt, outputs, nullptr, nullptr,
                       true, out);
}

extern "C" int vext_batch_create_adjoint(int n_systems, const vext_system *systems, int size,
                                         int n_axes, const double *axes,
                                         const vext_options *opt, float *const *energies,
                                         float *const *gradients, vext_batch *out) {
    if (!gradients) return fail(VEXT_ERR_ARGUMENT, "gradient outputs required");
    return batch_build(n_systems, systems, size, n_axes, axes, opt, energies, gradients, nullptr,
                       true, out);
}

namespace vext {

// Replay on exactly `stream` (0 = the legacy default stream).
int batch_replay(vext_batch b, cudaStream_t stream) {
    VEXT_CUDA(cudaGraphLaunch(b->exec, stream));
    return 0;
}

// Point system k's float32 energy / gradient outputs at `out` / `grad` for the
// replays that follow on `stream`: a stream-ordered update of the device copy
// of its BatchSys, which the captured kernels read at run time (no rebuild).
int batch_retarget(vext_batch b, int k, float *out, float *grad, cudaStream_t stream) {
    if (k < 0 || k >= (int)b->systems.size()) return fail(VEXT_ERR_ARGUMENT, "bad system index");
    if (!out || (b->adj && !grad)) return fail(VEXT_ERR_ARGUMENT, "null output");
    static_assert(offsetof(BatchSys, grad) == offsetof(BatchSys, out) + sizeof(float *),
                  "out and grad must be adjacent");
    float *ptrs[2] = {out, b->adj ? grad : nullptr};
    if (b->targets[k].first == ptrs[0] && b->targets[k].second == ptrs[1]) return 0;
    VEXT_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(b->d_sys + k) + offsetof(BatchSys, out),
                              ptrs, sizeof ptrs, cudaMemcpyHostToDevice, stream));
    b->targets[k] = {ptrs[0], ptrs[1]};
    return 0;
}

}  // namespace vext

extern "C" int vext_batch_run(vext_batch b, void *stream) {
    if (!b) return fail(VEXT_ERR_ARGUMENT, "null batch");
    return batch_replay(b, stream ? (cudaStream_t)stream : b->stream);
}

extern "C" int vext_batch_status(vext_batch b) {
    if (!b) return fail(VEXT_ERR_ARGUMENT, "null batch");
    int h[2] = {0, 0};
    VEXT_CUDA(cudaDeviceSynchronize());
    VEXT_CUDA(cudaMemcpy(&h[0], b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    VEXT_CUDA(cudaMemcpy(&h[1], b->d_refine, sizeof(int), cudaMemcpyDeviceToHost));
    if (h[0]) return fail(VEXT_ERR_TIMEOUT, "a device wait gave up (status %d)", h[0]);
    if (h[1] > b->refine_cap)
        return fail(VEXT_ERR_CAPACITY, "%d poses in the refinement band; %d refined", h[1],
                    b->refine_cap);
    return 0;
}

extern "C" int vext_batch_refined(vext_batch b, int64_t *poses) {
    if (!b || !poses) return fail(VEXT_ERR_ARGUMENT, "null batch or output");
    int h = 0;
    VEXT_CUDA(cudaDeviceSynchronize());
    VEXT_CUDA(cudaMemcpy(&h, b->d_refine, sizeof(int), cudaMemcpyDeviceToHost));
    *poses = std::min(h, b->refine_cap);
    return 0;
}

extern "C" int vext_batch_destroy(vext_batch b) {
    delete b;
    return 0;
}

extern "C" int vext_batch_tuning(vext_batch b, int max_candidates, int *n_candidates,
                                 int *shapes, int *grids, float *ms, const char **names) {
    if (!b) return fail(VEXT_ERR_ARGUMENT, "null batch");
    if (n_candidates) *n_candidates = b->n_cands;
    for (int c = 0; c < std::min(max_candidates, b->n_cands); ++c) {
        if (shapes) shapes[c] = b->cands[c].shape;
        if (grids) grids[c] = b->cands[c].grid;
        if (ms) ms[c] = b->tune_ms[c];
        if (names) names[c] = batch_kernel(b->kind, b->cands[c].shape).name;
    }
    return 0;
}

extern "C" int vext_batch_info(vext_batch b, int64_t *work_items, int64_t *poses,
                               int64_t *list_bytes, int *shape, int *grid) {
    if (!b) return fail(VEXT_ERR_ARGUMENT, "null batch");
    if (work_items) *work_items = b->n_items;
    if (poses) *poses = b->poses;
    if (list_bytes) *list_bytes = b->list_bytes;
    if (shape) *shape = b->config.shape;
    if (grid) *grid = b->config.grid;
    return 0;
}
