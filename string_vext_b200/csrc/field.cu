// Vext field kernels: every (grid center, director) pose of a size^3 grid.
//
// One CTA = one region (a block of CB grid centers) x one block of G*P
// directors; thread (cl, og) owns center cl and directors og + G p (p < P).
// The region's list streams through shared memory in kCH-entry chunks by
// bulk copies (stage.cuh); every staged entry is used by all 2P sites of all
// threads.  The pair loops live in pair.cuh.
//
// Precision: near entries (within r_split + max|offset| + rho of the origin)
// go through field_near_kernel in FP64 from the exact hi + lo positions; far
// entries through field_far_kernel in packed FP32x2 from hi, accumulated in
// FP32 over 16 entries and flushed into FP64.  Poses whose energy falls in
// the refinement band (where the 1e-6 relative criterion is tighter than the
// FP32 error) are recomputed in FP64 by refine_kernel.  With r_split =
// infinity every entry is near: field_near_kernel<..., 0> is then the FP64
// oracle kernel; plain_fp64_kernel is the straightforward FP64 baseline.
#include <algorithm>
#include <cmath>

#include <cuda.h>

#include "pair.cuh"

namespace vext {

constexpr int kPlainVariant = 1 << 20;
constexpr int kNaiveVariant = 1 << 21;

struct FieldArgs {
    Mat3 H;
    double rc2;
    float rc2f;
    double off0, off1;
    double floor_out2;        // |d0|^2 beyond which no site is inside a contact floor
    int S, O;
    const double *axes;       // device [O][3]
    const RegionInfo *regs;
    int n_regions;
    int bi, bj, bk, nrj, nrk; // region grid (for pose -> region)
    const float4 *hi, *lo;
    const float4 *tf;
    const double *td;
    int n_types;
    double *e64;              // [O][S^3]
    int *status;
};

__device__ __forceinline__ void center_of(const FieldArgs &a, const RegionInfo &r, int cl,
                                          int &gi, int &gj, int &gk) {
    const int lk = cl % r.nk, lj = (cl / r.nk) % r.nj, li = cl / (r.nk * r.nj);
    gi = r.i0 + li;
    gj = r.j0 + lj;
    gk = r.k0 + lk;
}

// Near pairs in FP64 over every region's near entries (all entries for the
// FP64 oracle region set); MODE as in near_chunk (pair.cuh).  Writes e64.
template <int CB, int G, int P, int MODE>
__global__ void __launch_bounds__(CB *G, 1) field_near_kernel(FieldArgs a) {
    constexpr int NT = CB * G;
    extern __shared__ __align__(128) unsigned char smem[];
    Stager st;
    st.bar = reinterpret_cast<uint64_t *>(smem);
    st.hib = reinterpret_cast<float4 *>(smem + 64);
    st.lob = st.hib + kStages * kCH;
    double *ed = reinterpret_cast<double *>(st.lob + kStages * kCH);   // [kCH][4]
    float4 *stf = reinterpret_cast<float4 *>(ed + 4 * kCH);
    double *std4 = reinterpret_cast<double *>(stf + a.n_types);

    const int tid = threadIdx.x;
    const RegionInfo r = a.regs[blockIdx.x];
    ChunkPlan plan;
    plan.init_range(r.off, r.n_near, r.n_near);
    load_types<NT>(stf, std4, a.tf, a.td, a.n_types);
    init_barriers(st);
    __syncthreads();
    stage_prologue(st, plan, a.hi, a.lo, 0);

    const int cl = tid % CB, og = tid / CB;
    const bool cvalid = cl < r.ni * r.nj * r.nk;
    int gi, gj, gk;
    center_of(a, r, cvalid ? cl : 0, gi, gj, gk);
    double cx, cy, cz;
    frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                 (gk + .5) / a.S - r.of[2], cx, cy, cz);
    const NearGeom g = near_geom(cx, cy, cz, a.off0, a.off1, a.rc2, a.floor_out2);
    const int obase = blockIdx.y * (G * P) + og;
    double shift_near = 0.0;
    double ux[P], uy[P], uz[P];
    double acc[P][2];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int o = min(obase + G * p, a.O - 1);
        ux[p] = a.axes[3 * o];
        uy[p] = a.axes[3 * o + 1];
        uz[p] = a.axes[3 * o + 2];
        acc[p][0] = acc[p][1] = 0.0;
    }
    for (int c = 0; c < plan.n_chunks; ++c) {
        if (!stage_wait(st, plan, c, 0, a.status)) return;
        int start, len;
        bool near;
        plan.chunk(c, start, len, near);
        const int s = c % kStages;
        near_convert<NT>(st.hib + s * kCH, st.lob + s * kCH, ed, len);
        __syncthreads();
        near_chunk<P, MODE>(ed, std4, len, g, ux, uy, uz, acc, shift_near);
        stage_next(st, plan, a.hi, a.lo, c, 0);
    }
    if (cvalid) {
        const size_t S3 = (size_t)a.S * a.S * a.S;
        const size_t cg = ((size_t)gi * a.S + gj) * a.S + gk;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int o = obase + G * p;
            if (o < a.O) a.e64[(size_t)o * S3 + cg] = acc[p][0] + acc[p][1] + 2.0 * shift_near;
        }
    }
}

// The earlier far kernel (far_chunk, pair.cuh: reciprocal of q^3 with a
// Newton step, every far entry masked), kept for comparison with
// field_far2_kernel.  A thread owns one grid center and P directors (lanes
// of a float2 = two directors); the far sums are added into e64 (written by
// the near kernel).
template <int CB, int G, int P, int MINB>
__global__ void __launch_bounds__(CB *G, MINB) field_far_kernel(FieldArgs a) {
    static_assert(P % 2 == 0, "directors are packed in pairs");
    constexpr int NT = CB * G, PP = P / 2;
    extern __shared__ __align__(128) unsigned char smem[];
    Stager st;
    st.bar = reinterpret_cast<uint64_t *>(smem);
    st.hib = reinterpret_cast<float4 *>(smem + 64);
    st.lob = st.hib;   // far chunks bring hi only
    float4 *stf = st.hib + kStages * kCH;

    const int tid = threadIdx.x;
    const RegionInfo r = a.regs[blockIdx.x];
    ChunkPlan plan;
    plan.init_range(r.off + r.n_near, 0, r.n_total - r.n_near);
    load_types<NT>(stf, nullptr, a.tf, a.td, a.n_types);
    init_barriers(st);
    __syncthreads();
    stage_prologue(st, plan, a.hi, a.lo, 0);

    const int cl = tid % CB, og = tid / CB;
    const bool cvalid = cl < r.ni * r.nj * r.nk;
    int gi, gj, gk;
    center_of(a, r, cvalid ? cl : 0, gi, gj, gk);
    double cxd, cyd, czd;
    frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                 (gk + .5) / a.S - r.of[2], cxd, cyd, czd);
    const FarGeom g = far_geom(cxd, cyd, czd, a.off0, a.off1, a.rc2f);
    const int obase = blockIdx.y * (G * P) + og;
    float2 ux[PP], uy[PP], uz[PP];
    double acc[P];
#pragma unroll
    for (int j = 0; j < PP; ++j) {
        const int o0 = min(obase + G * (2 * j), a.O - 1), o1 = min(obase + G * (2 * j + 1), a.O - 1);
        ux[j] = make_float2((float)a.axes[3 * o0], (float)a.axes[3 * o1]);
        uy[j] = make_float2((float)a.axes[3 * o0 + 1], (float)a.axes[3 * o1 + 1]);
        uz[j] = make_float2((float)a.axes[3 * o0 + 2], (float)a.axes[3 * o1 + 2]);
        acc[2 * j] = acc[2 * j + 1] = 0.0;
    }
    for (int c = 0; c < plan.n_chunks; ++c) {
        if (!stage_wait(st, plan, c, 0, a.status)) return;
        int start, len;
        bool near;
        plan.chunk(c, start, len, near);
        far_chunk<P, true, 16>(st.hib + (c % kStages) * kCH, stf, len, g, ux, uy, uz, acc);
        stage_next(st, plan, a.hi, a.lo, c, 0);
    }
    if (cvalid) {
        const size_t S3 = (size_t)a.S * a.S * a.S;
        const size_t cg = ((size_t)gi * a.S + gj) * a.S + gk;
#pragma unroll
        for (int j = 0; j < PP; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int o = obase + G * (2 * j + h);
                if (o < a.O) a.e64[(size_t)o * S3 + cg] += acc[2 * j + h];
            }
    }
}

// The default far kernel: far_chunk_fwd over the inner entries (no mask) and
// then the shell entries; same thread layout and output as field_far_kernel.
template <int CB, int G, int P, int MINB>
__global__ void __launch_bounds__(CB *G, MINB) field_far2_kernel(FieldArgs a) {
    constexpr int NT = CB * G, PP = P / 2;
    extern __shared__ __align__(128) unsigned char smem[];
    Stager st;
    st.bar = reinterpret_cast<uint64_t *>(smem);
    st.hib = reinterpret_cast<float4 *>(smem + 64);
    st.lob = st.hib;   // far chunks bring hi only
    float4 *stf = st.hib + kStages * kCH;

    const int tid = threadIdx.x;
    const RegionInfo r = a.regs[blockIdx.x];
    load_types<NT>(stf, nullptr, a.tf, a.td, a.n_types);
    init_barriers(st);
    __syncthreads();

    const int cl = tid % CB, og = tid / CB;
    const bool cvalid = cl < r.ni * r.nj * r.nk;
    int gi, gj, gk;
    center_of(a, r, cvalid ? cl : 0, gi, gj, gk);
    double cxd, cyd, czd;
    frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                 (gk + .5) / a.S - r.of[2], cxd, cyd, czd);
    const FarGeom g = far_geom(cxd, cyd, czd, a.off0, a.off1, a.rc2f);
    const int obase = blockIdx.y * (G * P) + og;
    float2 ux[PP], uy[PP], uz[PP];
    double acc[P];
#pragma unroll
    for (int j = 0; j < PP; ++j) {
        const int o0 = min(obase + G * (2 * j), a.O - 1), o1 = min(obase + G * (2 * j + 1), a.O - 1);
        ux[j] = make_float2((float)a.axes[3 * o0], (float)a.axes[3 * o1]);
        uy[j] = make_float2((float)a.axes[3 * o0 + 1], (float)a.axes[3 * o1 + 1]);
        uz[j] = make_float2((float)a.axes[3 * o0 + 2], (float)a.axes[3 * o1 + 2]);
        acc[2 * j] = acc[2 * j + 1] = 0.0;
    }
    double shift_sum = 0.0;
    unsigned seq = 0;
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {   // inner entries, then the shell
        ChunkPlan plan;
        plan.init_range(r.off + r.n_near + (pass ? r.n_inner : 0), 0,
                        pass ? r.n_total - r.n_near - r.n_inner : r.n_inner);
        stage_prologue(st, plan, a.hi, a.lo, seq);
        for (int c = 0; c < plan.n_chunks; ++c) {
            if (!stage_wait(st, plan, c, seq, a.status)) return;
            int start, len;
            bool near;
            plan.chunk(c, start, len, near);
            const float4 *hb = st.hib + ((seq + c) % kStages) * kCH;
            if (pass) far_chunk_fwd<P, 16, true>(hb, stf, len, g, ux, uy, uz, acc, shift_sum);
            else far_chunk_fwd<P, 16, false>(hb, stf, len, g, ux, uy, uz, acc, shift_sum);
            stage_next(st, plan, a.hi, a.lo, c, seq);
        }
        seq += plan.n_chunks;
    }
    if (cvalid) {
        const size_t S3 = (size_t)a.S * a.S * a.S;
        const size_t cg = ((size_t)gi * a.S + gj) * a.S + gk;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int o = obase + G * p;
            if (o < a.O) a.e64[(size_t)o * S3 + cg] += acc[p] + 2.0 * shift_sum;
        }
    }
}

// ---------------------------------------------------------------- epilogue

__global__ void flag_kernel(const double *e64, long long n, double lo, double hi, int *list) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = e64[i];
        if (v > lo && v < hi) {
            const int k = atomicAdd(&list[0], 1);
            list[1 + k] = (int)i;
        }
    }
}

// FP64 pair sum of one site against one region's list, lane-strided over a
// warp (no reduction here).
__device__ __forceinline__ double site_sum_fp64(const FieldArgs &a, const RegionInfo &r,
                                                double px, double py, double pz, int lane) {
    double sum = 0.0;
    for (int e = lane; e < r.n_total; e += 32) {
        const float4 h = a.hi[r.off + e], l = a.lo[r.off + e];
        const double dx = px - ((double)h.x + (double)l.x);
        const double dy = py - ((double)h.y + (double)l.y);
        const double dz = pz - ((double)h.z + (double)l.z);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < a.rc2) {
            const int t = __float_as_int(h.w);
            const double c12 = a.td[4 * t], c6 = a.td[4 * t + 1], shift = a.td[4 * t + 2],
                         fl = a.td[4 * t + 3];
            const double s2 = d2 < fl ? fl : d2;
            const double i2 = 1.0 / s2;
            const double i6 = i2 * i2 * i2;
            sum += c12 * i6 * i6 - c6 * i6 + shift;
        }
    }
    return sum;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int region_of(const FieldArgs &a, int gi, int gj, int gk) {
    return ((gi / a.bi) * a.nrj + gj / a.bj) * a.nrk + gk / a.bk;
}

__global__ void refine_kernel(FieldArgs a, const int *list) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int count = list[0];
    const long long S3 = (long long)a.S * a.S * a.S;
    for (int q = warp; q < count; q += nwarps) {
        const long long idx = list[1 + q];
        const int o = (int)(idx / S3);
        const long long c = idx % S3;
        const int gi = (int)(c / ((long long)a.S * a.S)), gj = (int)((c / a.S) % a.S),
                  gk = (int)(c % a.S);
        const RegionInfo r = a.regs[region_of(a, gi, gj, gk)];
        double cx, cy, cz;
        frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                     (gk + .5) / a.S - r.of[2], cx, cy, cz);
        const double ux = a.axes[3 * o], uy = a.axes[3 * o + 1], uz = a.axes[3 * o + 2];
        double e = site_sum_fp64(a, r, cx + a.off0 * ux, cy + a.off0 * uy, cz + a.off0 * uz, lane);
        e += site_sum_fp64(a, r, cx + a.off1 * ux, cy + a.off1 * uy, cz + a.off1 * uz, lane);
        e = warp_sum(e);
        if (lane == 0) a.e64[idx] = e;
    }
}

// Single-site field at the grid centers (site 0 parameters, no offset):
// the reference's site_K (src/string_vext/vext.py:27-29, 33).
__global__ void site_kernel(FieldArgs a, float *site_K) {
    const int lane = threadIdx.x & 31;
    const long long S3 = (long long)a.S * a.S * a.S;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < S3;
         c += nwarps) {
        const int gi = (int)(c / ((long long)a.S * a.S)), gj = (int)((c / a.S) % a.S),
                  gk = (int)(c % a.S);
        const RegionInfo r = a.regs[region_of(a, gi, gj, gk)];
        double cx, cy, cz;
        frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                     (gk + .5) / a.S - r.of[2], cx, cy, cz);
        const double e = warp_sum(site_sum_fp64(a, r, cx, cy, cz, lane));
        if (lane == 0) {
            site_K[c] = (float)e;
            site_K[S3 + c] = (float)e;
        }
    }
}

// Per center: float32 orientation field, marginal -T (logsumexp(-E/T) - log O)
// (physics.py:126-130) and grid = asinh(marginal / 1000) (vext.py:40).
__global__ void finalize_kernel(const double *e64, int S, int O, double T, float *orientation_K,
                                float *marginal_K, float *grid, int *nonfinite) {
    const long long S3 = (long long)S * S * S;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < S3;
         c += (long long)gridDim.x * blockDim.x) {
        double amax = -INFINITY;
        bool finite = true;
        for (int o = 0; o < O; ++o) {
            const double e = e64[(long long)o * S3 + c];
            finite = finite && isfinite(e);
            if (orientation_K) orientation_K[(long long)o * S3 + c] = (float)e;
            amax = fmax(amax, -e / T);
        }
        if (!finite) {
            atomicAdd(nonfinite, 1);
            continue;
        }
        if (marginal_K || grid) {
            double sum = 0.0;
            for (int o = 0; o < O; ++o) sum += exp(-e64[(long long)o * S3 + c] / T - amax);
            const double m = -T * (log(sum) + amax - log((double)O));
            const float m32 = (float)m;
            if (marginal_K) marginal_K[c] = m32;
            if (grid) grid[c] = (float)asinh((double)(m32 / 1000.0f));
        }
    }
}

// [O][S^3] -> [S^3][O] (the reference's (n_centers, n_axes) FP64 array).
__global__ void transpose_kernel(const double *e64, long long S3, int O, double *out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < S3 * O;
         i += (long long)gridDim.x * blockDim.x) {
        const long long c = i / O;
        const int o = (int)(i % O);
        out[i] = e64[(long long)o * S3 + c];
    }
}

// Exact FP64 count of in-cutoff (site, image) pairs over the whole field:
// the algorithmic unit of work.  One warp per grid center, lanes over the
// region's entries, every director and both sites tested per entry.
__global__ void count_kernel(FieldArgs a, unsigned long long *total) {
    const int lane = threadIdx.x & 31;
    const long long S3 = (long long)a.S * a.S * a.S;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long mine = 0, far = 0;
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < S3;
         c += nwarps) {
        const int gi = (int)(c / ((long long)a.S * a.S)), gj = (int)((c / a.S) % a.S),
                  gk = (int)(c % a.S);
        const RegionInfo r = a.regs[region_of(a, gi, gj, gk)];
        double cx, cy, cz;
        frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                     (gk + .5) / a.S - r.of[2], cx, cy, cz);
        for (int e = lane; e < r.n_total; e += 32) {
            const float4 h = a.hi[r.off + e], l = a.lo[r.off + e];
            const double x = (double)h.x + (double)l.x, y = (double)h.y + (double)l.y,
                         z = (double)h.z + (double)l.z;
            for (int o = 0; o < a.O; ++o) {
                const double ux = a.axes[3 * o], uy = a.axes[3 * o + 1], uz = a.axes[3 * o + 2];
                for (int s = 0; s < 2; ++s) {
                    const double off = s ? a.off1 : a.off0;
                    const double dx = cx + off * ux - x, dy = cy + off * uy - y,
                                 dz = cz + off * uz - z;
                    const bool in = (dx * dx + dy * dy + dz * dz) < a.rc2;
                    mine += in;
                    far += in && e >= r.n_near;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mine += __shfl_xor_sync(0xffffffffu, mine, o);
        far += __shfl_xor_sync(0xffffffffu, far, o);
    }
    if (lane == 0) {
        atomicAdd(total, mine);
        atomicAdd(total + 1, far);
    }
}

// The plain FP64 baseline: one thread per pose, both sites, every entry of
// its region read straight from global memory (hi + lo), IEEE division, no
// staging, no register blocking -- the straightforward one-field-per-launch
// FP64 kernel the tiled kernels are measured against.
__global__ void __launch_bounds__(256) plain_fp64_kernel(FieldArgs a) {
    const long long S3 = (long long)a.S * a.S * a.S;
    const long long n = S3 * a.O;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long c = idx % S3;   // consecutive threads: consecutive centers
        const int o = (int)(idx / S3);
        const int gi = (int)(c / ((long long)a.S * a.S)), gj = (int)((c / a.S) % a.S),
                  gk = (int)(c % a.S);
        const RegionInfo r = a.regs[region_of(a, gi, gj, gk)];
        double cx, cy, cz;
        frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                     (gk + .5) / a.S - r.of[2], cx, cy, cz);
        const double ux = a.axes[3 * o], uy = a.axes[3 * o + 1], uz = a.axes[3 * o + 2];
        double e = 0.0;
        for (int s = 0; s < 2; ++s) {
            const double off = s ? a.off1 : a.off0;
            const double px = cx + off * ux, py = cy + off * uy, pz = cz + off * uz;
            for (int k = 0; k < r.n_total; ++k) {
                const float4 h = a.hi[r.off + k], l = a.lo[r.off + k];
                const double dx = px - ((double)h.x + (double)l.x);
                const double dy = py - ((double)h.y + (double)l.y);
                const double dz = pz - ((double)h.z + (double)l.z);
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 >= a.rc2) continue;
                const int t = __float_as_int(h.w);
                const double fl = a.td[4 * t + 3];
                const double s2 = d2 < fl ? fl : d2;
                const double i2 = 1.0 / s2;
                const double i6 = i2 * i2 * i2;
                e += a.td[4 * t] * i6 * i6 - a.td[4 * t + 1] * i6 + a.td[4 * t + 2];
            }
        }
        a.e64[idx] = e;
    }
}

// The naive FP32 field (precision study): plain_fp64_kernel's loop in FP32 --
// sites relative to the region origin rounded to FP32, entries from hi only,
// IEEE FP32 division, one FP32 sum per pose over both sites.
__global__ void __launch_bounds__(256) plain_fp32_kernel(FieldArgs a) {
    const long long S3 = (long long)a.S * a.S * a.S;
    const long long n = S3 * a.O;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long c = idx % S3;
        const int o = (int)(idx / S3);
        const int gi = (int)(c / ((long long)a.S * a.S)), gj = (int)((c / a.S) % a.S),
                  gk = (int)(c % a.S);
        const RegionInfo r = a.regs[region_of(a, gi, gj, gk)];
        double cx, cy, cz;
        frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                     (gk + .5) / a.S - r.of[2], cx, cy, cz);
        const double ux = a.axes[3 * o], uy = a.axes[3 * o + 1], uz = a.axes[3 * o + 2];
        float e = 0.f;
        for (int s = 0; s < 2; ++s) {
            const double off = s ? a.off1 : a.off0;
            const float px = (float)(cx + off * ux), py = (float)(cy + off * uy),
                        pz = (float)(cz + off * uz);
            for (int k = 0; k < r.n_total; ++k) {
                const float4 h = a.hi[r.off + k];
                const float dx = px - h.x, dy = py - h.y, dz = pz - h.z;
                const float d2 = dx * dx + dy * dy + dz * dz;
                if (d2 >= a.rc2f) continue;
                const float4 tp = a.tf[__float_as_int(h.w)];   // (c12, c6, shift, floor2)
                const float s2 = d2 < tp.w ? tp.w : d2;
                const float i2 = 1.0f / s2;
                const float i6 = i2 * i2 * i2;
                e += tp.x * i6 * i6 - tp.y * i6 + tp.z;
            }
        }
        a.e64[idx] = (double)e;
    }
}

// The plain FP64 forward + adjoint: plain_fp64_kernel plus, per in-cutoff
// pair off the contact floor, dE/d(r^2) = (-6 c12 i6^2 + 3 c6 i6) i2 and the
// site gradient 2 dE/d(r^2) (site - x); dE/dc = sum over sites, dE/du =
// sum o_s x site gradient, projected on the plane normal to u.  Any output
// may be null ([O][S^3] energies, [O][S^3][6] gradients).
__global__ void __launch_bounds__(256)
    plain_fp64_adj_kernel(FieldArgs a, double *e64, double *g64, float *e32, float *g32) {
    const long long S3 = (long long)a.S * a.S * a.S;
    const long long n = S3 * a.O;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long c = idx % S3;
        const int o = (int)(idx / S3);
        const int gi = (int)(c / ((long long)a.S * a.S)), gj = (int)((c / a.S) % a.S),
                  gk = (int)(c % a.S);
        const RegionInfo r = a.regs[region_of(a, gi, gj, gk)];
        double cx, cy, cz;
        frac_to_cart(a.H, (gi + .5) / a.S - r.of[0], (gj + .5) / a.S - r.of[1],
                     (gk + .5) / a.S - r.of[2], cx, cy, cz);
        const double u[3] = {a.axes[3 * o], a.axes[3 * o + 1], a.axes[3 * o + 2]};
        double e = 0.0, g[6];
        fp64_pose_pairs(a.hi, a.lo, a.td, r.off, r.n_total, 0, 1, a.rc2, a.off0, a.off1, cx, cy,
                        cz, u, e, g);
        fp64_tangent(u, g);
        if (e64) e64[idx] = e;
        if (e32) e32[idx] = (float)e;
        for (int k = 0; k < 6; ++k) {
            if (g64) g64[6 * idx + k] = g[k];
            if (g32) g32[6 * idx + k] = (float)g[k];
        }
    }
}

// ---------------------------------------------------------------- launchers

static size_t near_smem(int n_types) {
    return kStageBytes + (size_t)kCH * 4 * sizeof(double) + (size_t)n_types * (16 + 32);
}

static size_t far_smem(int n_types) {
    return 64 + (size_t)kStages * kCH * sizeof(float4) + (size_t)n_types * 16;
}

template <typename K>
static int launch_t(K kern, dim3 grid, int threads, size_t smem, const FieldArgs &a,
                    cudaStream_t stream) {
    VEXT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, threads, smem, stream>>>(a);
    VEXT_CUDA(cudaGetLastError());
    return 0;
}

// Near (FP64) kernel over every region.  mode 0 = the FP64 oracle kernel
// (must run on an all-near region set), 1 = mixed with cutoff test, 2 =
// mixed without (near pairs provably inside the cutoff).
static int launch_near(const FieldArgs &a, int cb, int mode, cudaStream_t stream) {
    const size_t smem = near_smem(a.n_types);
    if (cb == 32) {
        dim3 grid(a.n_regions, (a.O + 31) / 32);
        if (mode == 0) return launch_t(field_near_kernel<32, 8, 4, 0>, grid, 256, smem, a, stream);
        if (mode == 1) return launch_t(field_near_kernel<32, 8, 4, 1>, grid, 256, smem, a, stream);
        return launch_t(field_near_kernel<32, 8, 4, 2>, grid, 256, smem, a, stream);
    }
    dim3 grid(a.n_regions, (a.O + 63) / 64);
    if (cb == 8) {
        if (mode == 0) return launch_t(field_near_kernel<8, 16, 4, 0>, grid, 128, smem, a, stream);
        if (mode == 1) return launch_t(field_near_kernel<8, 16, 4, 1>, grid, 128, smem, a, stream);
        return launch_t(field_near_kernel<8, 16, 4, 2>, grid, 128, smem, a, stream);
    }
    if (mode == 0) return launch_t(field_near_kernel<16, 16, 4, 0>, grid, 256, smem, a, stream);
    if (mode == 1) return launch_t(field_near_kernel<16, 16, 4, 1>, grid, 256, smem, a, stream);
    return launch_t(field_near_kernel<16, 16, 4, 2>, grid, 256, smem, a, stream);
}

// Far kernels (threads = CB x G, directors per CTA = G x P):
//   default: field_far2_kernel <16, 8, 4> (16-center regions, 32 directors
//            per CTA; <8, 16, 4> with 64 directors for 8-center regions,
//            <32, 8, 4> for 32), 6 CTAs/SM of 128: inner entries without the
//            cutoff mask, reciprocal of q per lane cubed, no Newton step
//   9:       field_far_kernel <16, 8, 4>: reciprocal of q^3 per lane + Newton
//            step, every entry masked (the earlier kernel, for comparison)
static int launch_far(const FieldArgs &a, int cb, int variant, cudaStream_t stream) {
    const size_t smem = far_smem(a.n_types);
    if (cb == 8)
        return launch_t(field_far2_kernel<8, 16, 4, 6>, dim3(a.n_regions, (a.O + 63) / 64), 128,
                        smem, a, stream);
    const dim3 grid(a.n_regions, (a.O + 31) / 32);
    if (cb == 32) return launch_t(field_far2_kernel<32, 8, 4, 2>, grid, 256, smem, a, stream);
    if (variant == 9) return launch_t(field_far_kernel<16, 8, 4, 4>, grid, 128, smem, a, stream);
    return launch_t(field_far2_kernel<16, 8, 4, 6>, grid, 128, smem, a, stream);
}

static FieldArgs make_args(System *sys, const RegionSet *rs, int n_axes, const double *d_axes,
                           double *d_e64) {
    FieldArgs a;
    a.H = sys->H;
    a.rc2 = sys->cutoff * sys->cutoff;
    a.rc2f = (float)a.rc2;
    a.off0 = sys->offsets[0];
    a.floor_out2 = floor_clear_radius2(*sys);
    a.off1 = sys->offsets[1];
    a.S = rs->size;
    a.O = n_axes;
    a.axes = d_axes;
    a.regs = rs->d_info;
    a.n_regions = rs->n_regions;
    a.bi = rs->bi;
    a.bj = rs->bj;
    a.bk = rs->bk;
    a.nrj = rs->n_rj;
    a.nrk = rs->n_rk;
    a.hi = rs->d_hi;
    a.lo = rs->d_lo;
    a.tf = sys->d_tf;
    a.td = sys->d_td;
    a.n_types = sys->n_types;
    a.e64 = d_e64;
    a.status = sys->d_status;
    return a;
}

// The near kernel writes e64, the far kernel adds its sums to it.
int launch_field(System *sys, const RegionSet *rs, int n_axes, const double *d_axes,
                 double *d_e64, int cb, int variant, cudaStream_t stream) {
    FieldArgs a = make_args(sys, rs, n_axes, d_axes, d_e64);
    sys->split_timed = false;
    if (rs->r_split >= 1e29 && variant == kPlainVariant) {            // plain FP64 baseline
        plain_fp64_kernel<<<148 * 16, 256, 0, stream>>>(a);
        VEXT_CUDA(cudaGetLastError());
        return 0;
    }
    if (rs->r_split >= 1e29 && variant == kNaiveVariant) {            // naive FP32 (study)
        plain_fp32_kernel<<<148 * 16, 256, 0, stream>>>(a);
        VEXT_CUDA(cudaGetLastError());
        return 0;
    }
    if (rs->r_split >= 1e29) return launch_near(a, cb, 0, stream);   // FP64 oracle
    // near pairs are at most r_split + 2 (rho + max|offset|) apart
    double rho = 0;
    for (const RegionInfo &r : rs->h_info) rho = std::max(rho, r.rho);
    const int near_mode = rs->r_split + 2.0 * (rho + sys->max_offset) + 1e-6 < sys->cutoff ? 2 : 1;
    VEXT_TRY(launch_near(a, cb, near_mode, stream));
    VEXT_CUDA(cudaEventRecord(sys->ev[5], stream));   // near | far split of the timing
    sys->split_timed = true;
    return launch_far(a, cb, variant, stream);
}

// Everything on device pointers and `stream`; region lists are built (with
// a host synchronisation) on first use of (size, shape, r_split).
static int field_device(System *sys, int size, int n_axes, const double *axes_host,
                        const Options &o, float *d_oK, double *d_e64_out, float *d_marg,
                        float *d_site, float *d_grid, cudaStream_t stream,
                        vext_field_stats *stats) {
    if (size < 1 || n_axes < 1 || !axes_host)
        return fail(VEXT_ERR_ARGUMENT, "size >= 1, n_axes >= 1 and axes required");
    const long long S3 = (long long)size * size * size;
    if (S3 * n_axes >= (1LL << 31) - 1)
        return fail(VEXT_ERR_CAPACITY, "size^3 * n_axes must stay below 2^31");
    for (int k = 0; k < 3 * n_axes; ++k)
        if (!std::isfinite(axes_host[k])) return fail(VEXT_ERR_ARGUMENT, "non-finite director");
    if (o.mode != VEXT_MODE_MIXED && o.mode != VEXT_MODE_FP64 && o.mode != VEXT_MODE_FP64_PLAIN &&
        o.mode != VEXT_MODE_FP32_NAIVE)
        return fail(VEXT_ERR_ARGUMENT, "unknown precision mode %d", o.mode);
    const bool fp64 = o.mode != VEXT_MODE_MIXED;   // all-entry region lists
    // regions of 16 grid centers by default (8 or 32 on request; 8 only in the
    // mixed mode): a call that builds its lists pays twice the list work on
    // 8-center regions for 5 % less pair work, so 16 stays the default here
    const int cb = o.cb == 32 ? 32 : o.cb == 8 && !fp64 ? 8 : 16;
    const double r_split = fp64 ? 1e30 : o.r_split;
    RegionSet *rs = nullptr;
    VEXT_TRY(get_field_regions(sys, size, cb, r_split, &rs, stream));
    const size_t n = (size_t)S3 * n_axes;
    VEXT_TRY(ensure_capacity(sys->d_axes, sys->axes_cap, 3 * (size_t)n_axes));
    VEXT_TRY(ensure_capacity(sys->d_e64, sys->e64_cap, n));
    VEXT_TRY(ensure_capacity(sys->d_refine, sys->refine_cap, n + 1));
    VEXT_TRY(ensure_capacity(sys->d_flags, sys->flags_cap, 4));
    VEXT_CUDA(cudaMemcpyAsync(sys->d_axes, axes_host, sizeof(double) * 3 * n_axes,
                              cudaMemcpyHostToDevice, stream));
    VEXT_CUDA(cudaMemsetAsync(sys->d_flags, 0, sizeof(int) * 4, stream));
    VEXT_CUDA(cudaMemsetAsync(sys->d_refine, 0, sizeof(int), stream));
    const FieldArgs a = make_args(sys, rs, n_axes, sys->d_axes, sys->d_e64);
    VEXT_CUDA(cudaEventRecord(sys->ev[0], stream));
    VEXT_TRY(launch_field(sys, rs, n_axes, sys->d_axes, sys->d_e64, cb,
                          o.mode == VEXT_MODE_FP64_PLAIN   ? kPlainVariant
                          : o.mode == VEXT_MODE_FP32_NAIVE ? kNaiveVariant
                                                           : o.variant,
                          stream));
    VEXT_CUDA(cudaEventRecord(sys->ev[1], stream));
    if (o.mode == VEXT_MODE_MIXED && o.band_hi > o.band_lo) {
        flag_kernel<<<592, 256, 0, stream>>>(sys->d_e64, (long long)n, o.band_lo, o.band_hi,
                                              sys->d_refine);
        VEXT_CUDA(cudaGetLastError());
        refine_kernel<<<1184, 256, 0, stream>>>(a, sys->d_refine);
        VEXT_CUDA(cudaGetLastError());
    }
    if (d_site) {
        site_kernel<<<1184, 256, 0, stream>>>(a, d_site);
        VEXT_CUDA(cudaGetLastError());
    }
    finalize_kernel<<<592, 256, 0, stream>>>(sys->d_e64, size, n_axes, sys->temperature, d_oK,
                                              d_marg, d_grid, sys->d_flags);
    VEXT_CUDA(cudaGetLastError());
    if (d_e64_out) {
        transpose_kernel<<<1184, 256, 0, stream>>>(sys->d_e64, S3, n_axes, d_e64_out);
        VEXT_CUDA(cudaGetLastError());
    }
    VEXT_CUDA(cudaEventRecord(sys->ev[2], stream));
    sys->timed = true;
    if (stats) {
        VEXT_CUDA(cudaEventSynchronize(sys->ev[2]));
        float k_ms = 0, e_ms = 0;
        VEXT_CUDA(cudaEventElapsedTime(&k_ms, sys->ev[0], sys->ev[1]));
        VEXT_CUDA(cudaEventElapsedTime(&e_ms, sys->ev[1], sys->ev[2]));
        int refined = 0;
        VEXT_CUDA(cudaMemcpy(&refined, sys->d_refine, sizeof(int), cudaMemcpyDeviceToHost));
        stats->poses = (int64_t)n;
        stats->regions = rs->n_regions;
        stats->list_entries = rs->n_entries;
        stats->near_entries = rs->n_near;
        stats->outer_entries = rs->n_outer;
        stats->refined_poses = o.mode == VEXT_MODE_MIXED && o.band_hi > o.band_lo ? refined : 0;
        stats->list_build_ms = rs->build_ms;
        stats->kernel_ms = k_ms;
        stats->epilogue_ms = e_ms;
    }
    return 0;
}

static int check_nonfinite(System *sys, cudaStream_t stream) {
    int h[2] = {0, 0};
    VEXT_CUDA(cudaMemcpyAsync(h, sys->d_flags, sizeof(int), cudaMemcpyDeviceToHost, stream));
    VEXT_CUDA(cudaStreamSynchronize(stream));
    if (h[0]) return fail(VEXT_ERR_NONFINITE, "%d grid centers with a non-finite energy", h[0]);
    return check_status(sys, stream);
}

}  // namespace vext

using namespace vext;

extern "C" int vext_field(vext_system h, int size, int n_axes, const double *axes,
                          const vext_options *opt, float *orientation_K, double *energy_f64,
                          float *marginal_K, float *site_K, float *grid, vext_field_stats *stats) {
    if (!h) return fail(VEXT_ERR_ARGUMENT, "null system");
    System *sys = &h->sys;
    std::lock_guard<std::mutex> guard(sys->lock);
    VEXT_CUDA(cudaSetDevice(sys->device));
    const Options o = resolve_options(opt);
    const size_t S3 = (size_t)size * size * size, n = S3 * (size_t)(n_axes > 0 ? n_axes : 0);
    cudaStream_t st = sys->stream;
    if (orientation_K) VEXT_TRY(ensure_capacity(sys->d_f32, sys->f32_cap, n));
    if (marginal_K || site_K || grid) VEXT_TRY(ensure_capacity(sys->d_small, sys->small_cap, 4 * S3));
    if (energy_f64) VEXT_TRY(ensure_capacity(sys->d_e64T, sys->e64T_cap, n));
    float *dm = marginal_K ? sys->d_small : nullptr;
    float *ds = site_K ? sys->d_small + S3 : nullptr;
    float *dg = grid ? sys->d_small + 3 * S3 : nullptr;
    vext_field_stats local;
    VEXT_TRY(field_device(sys, size, n_axes, axes, o, orientation_K ? sys->d_f32 : nullptr,
                          energy_f64 ? sys->d_e64T : nullptr, dm, ds, dg, st,
                          stats ? stats : &local));
    if (orientation_K)
        VEXT_CUDA(cudaMemcpyAsync(orientation_K, sys->d_f32, sizeof(float) * n,
                                  cudaMemcpyDeviceToHost, st));
    if (energy_f64)
        VEXT_CUDA(cudaMemcpyAsync(energy_f64, sys->d_e64T, sizeof(double) * n,
                                  cudaMemcpyDeviceToHost, st));
    if (marginal_K)
        VEXT_CUDA(cudaMemcpyAsync(marginal_K, dm, sizeof(float) * S3, cudaMemcpyDeviceToHost, st));
    if (site_K)
        VEXT_CUDA(cudaMemcpyAsync(site_K, ds, sizeof(float) * 2 * S3, cudaMemcpyDeviceToHost, st));
    if (grid) VEXT_CUDA(cudaMemcpyAsync(grid, dg, sizeof(float) * S3, cudaMemcpyDeviceToHost, st));
    return check_nonfinite(sys, st);
}

extern "C" int vext_field_device(vext_system h, int size, int n_axes, const double *axes_host,
                                 const vext_options *opt, float *orientation_K,
                                 double *energy_f64, float *marginal_K, float *site_K,
                                 float *grid, void *stream) {
    if (!h) return fail(VEXT_ERR_ARGUMENT, "null system");
    System *sys = &h->sys;
    std::lock_guard<std::mutex> guard(sys->lock);
    VEXT_CUDA(cudaSetDevice(sys->device));
    const Options o = resolve_options(opt);
    return field_device(sys, size, n_axes, axes_host, o, orientation_K, energy_f64, marginal_K,
                        site_K, grid, (cudaStream_t)stream, nullptr);
}

namespace vext {

// Cache key of the options that shape a batch (kernel table, pinned shape,
// region size).
static double batch_key(const Options &o) {
    return o.variant + 65536.0 * o.batch_shape + 16777216.0 * o.cb;
}

static int field_adjoint_device(vext_system h, int size, int n_axes, const double *axes,
                                const Options &o, const vext_options *opt, float *energy,
                                float *gradient, double *energy_f64, double *gradient_f64,
                                cudaStream_t stream) {
    System *sys = &h->sys;
    if (size < 1 || n_axes < 1 || !axes)
        return fail(VEXT_ERR_ARGUMENT, "size >= 1, n_axes >= 1 and axes required");
    const long long S3 = (long long)size * size * size;
    if (S3 * n_axes * 6 >= (1LL << 40))
        return fail(VEXT_ERR_CAPACITY, "field too large");
    for (int k = 0; k < 3 * n_axes; ++k)
        if (!std::isfinite(axes[k])) return fail(VEXT_ERR_ARGUMENT, "non-finite director");
    if (o.mode == VEXT_MODE_MIXED) {
        if (!energy || !gradient)
            return fail(VEXT_ERR_ARGUMENT, "the mixed adjoint writes float32 energy and gradient");
        if (gradient_f64)
            return fail(VEXT_ERR_ARGUMENT, "the FP64 gradient needs an FP64 mode");
        const bool same = sys->adj_batch && sys->adj_size == size &&
                          sys->adj_axes.size() == 3 * (size_t)n_axes &&
                          std::equal(axes, axes + 3 * n_axes, sys->adj_axes.begin()) &&
                          sys->adj_key[0] == o.r_split && sys->adj_key[1] == o.band_lo &&
                          sys->adj_key[2] == o.band_hi &&
                          sys->adj_key[3] == batch_key(o) &&
                          sys->adj_energy64 == energy_f64;
        if (!same) {
            if (sys->adj_batch) vext_batch_destroy(sys->adj_batch);   // (host parts stay)
            sys->adj_batch = nullptr;
            vext_batch b = nullptr;
            VEXT_TRY(batch_build(1, &h, size, n_axes, axes, opt, &energy, &gradient,
                                 energy_f64 ? &energy_f64 : nullptr, false, &b));
            sys->adj_batch = b;
            sys->adj_size = size;
            sys->adj_axes.assign(axes, axes + 3 * n_axes);
            sys->adj_key[0] = o.r_split;
            sys->adj_key[1] = o.band_lo;
            sys->adj_key[2] = o.band_hi;
            sys->adj_key[3] = batch_key(o);
            sys->adj_energy64 = energy_f64;
        }
        // other float32 outputs than the last call's: a stream-ordered update
        // of the batch's output pointers, no rebuild
        VEXT_TRY(batch_retarget(sys->adj_batch, 0, energy, gradient, stream));
        return batch_replay(sys->adj_batch, stream);
    }
    if (o.mode != VEXT_MODE_FP64 && o.mode != VEXT_MODE_FP64_PLAIN)
        return fail(VEXT_ERR_ARGUMENT, "unknown precision mode %d", o.mode);
    RegionSet *rs = nullptr;
    VEXT_TRY(get_field_regions(sys, size, 16, 1e30, &rs, stream));
    VEXT_TRY(ensure_capacity(sys->d_axes, sys->axes_cap, 3 * (size_t)n_axes));
    VEXT_CUDA(cudaMemcpyAsync(sys->d_axes, axes, sizeof(double) * 3 * n_axes,
                              cudaMemcpyHostToDevice, stream));
    const FieldArgs a = make_args(sys, rs, n_axes, sys->d_axes, nullptr);
    plain_fp64_adj_kernel<<<148 * 16, 256, 0, stream>>>(a, energy_f64, gradient_f64, energy,
                                                        gradient);
    VEXT_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace vext

extern "C" int vext_field_adjoint_device(vext_system h, int size, int n_axes,
                                         const double *axes_host, const vext_options *opt,
                                         float *energy, float *gradient, double *energy_f64,
                                         double *gradient_f64, void *stream) {
    if (!h) return fail(VEXT_ERR_ARGUMENT, "null system");
    System *sys = &h->sys;
    std::lock_guard<std::mutex> guard(sys->lock);
    VEXT_CUDA(cudaSetDevice(sys->device));
    const Options o = resolve_options(opt);
    return field_adjoint_device(h, size, n_axes, axes_host, o, opt, energy, gradient, energy_f64,
                                gradient_f64, (cudaStream_t)stream);
}

// Device address of host memory the kernels may write directly: [p, p +
// bytes) must lie inside one page-locked, device-mapped allocation (checked
// by the driver's allocation range of p and by the mapping of the last byte);
// otherwise null, and the caller copies through device memory instead.
static void *mapped_host_range(void *p, size_t bytes) {
    using RangeFn = CUresult (*)(void *, CUpointer_attribute, CUdeviceptr);
    static RangeFn range_fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (RangeFn) nullptr;
        }
        return reinterpret_cast<RangeFn>(f);
    }();
    if (!range_fn || !p || bytes == 0) return nullptr;
    cudaPointerAttributes first, last;
    if (cudaPointerGetAttributes(&first, p) != cudaSuccess ||
        cudaPointerGetAttributes(&last, static_cast<char *>(p) + bytes - 1) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (first.type != cudaMemoryTypeHost || last.type != cudaMemoryTypeHost ||
        !first.devicePointer ||
        static_cast<char *>(last.devicePointer) !=
            static_cast<char *>(first.devicePointer) + (bytes - 1))
        return nullptr;
    const CUdeviceptr d = reinterpret_cast<CUdeviceptr>(first.devicePointer);
    CUdeviceptr start = 0;
    size_t range = 0;
    if (range_fn(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, d) != CUDA_SUCCESS ||
        range_fn(&range, CU_POINTER_ATTRIBUTE_RANGE_SIZE, d) != CUDA_SUCCESS)
        return nullptr;
    if (d < start || d - start > range || bytes > range - (d - start)) return nullptr;
    return first.devicePointer;
}

extern "C" int vext_field_adjoint(vext_system h, int size, int n_axes, const double *axes,
                                  const vext_options *opt, float *energy, float *gradient) {
    if (!h) return fail(VEXT_ERR_ARGUMENT, "null system");
    if (!energy || !gradient) return fail(VEXT_ERR_ARGUMENT, "energy and gradient required");
    if (size < 1 || n_axes < 1) return fail(VEXT_ERR_ARGUMENT, "size >= 1 and n_axes >= 1");
    System *sys = &h->sys;
    std::lock_guard<std::mutex> guard(sys->lock);
    VEXT_CUDA(cudaSetDevice(sys->device));
    const Options o = resolve_options(opt);
    const size_t n = (size_t)size * size * size * (size_t)n_axes;
    VEXT_TRY(ensure_capacity(sys->d_f32, sys->f32_cap, n));
    VEXT_TRY(ensure_capacity(sys->d_g32, sys->g32_cap, 6 * n));
    cudaStream_t st = sys->stream;
    if (o.mode == VEXT_MODE_MIXED) {
        // page-locked host outputs: one batch over all directors writes the
        // float32 results straight into them (the transfer runs beside the
        // pair work)
        float *de = static_cast<float *>(mapped_host_range(energy, sizeof(float) * n));
        float *dg = de ? static_cast<float *>(mapped_host_range(gradient, sizeof(float) * 6 * n))
                       : nullptr;
        if (de && dg) {
            VEXT_TRY(field_adjoint_device(h, size, n_axes, axes, o, opt, de, dg, nullptr, nullptr,
                                          st));
            VEXT_CUDA(cudaStreamSynchronize(st));
            return vext_batch_status(sys->adj_batch);
        }
    }
    if (o.mode == VEXT_MODE_MIXED) {
        // pageable host outputs: one batch per block of the batch's work-item
        // directors (64 by default); block k's copy (on aux) overlaps block
        // k + 1's pair work (on st)
        for (int k = 0; k < 3 * n_axes; ++k)
            if (!std::isfinite(axes[k])) return fail(VEXT_ERR_ARGUMENT, "non-finite director");
        const size_t S3 = (size_t)size * size * size;
        const int blk = batch_item_directors(o, true), parts = (n_axes + blk - 1) / blk;
        const bool same = (int)sys->host_parts.size() == parts && sys->host_size == size &&
                          sys->host_axes.size() == 3 * (size_t)n_axes &&
                          std::equal(axes, axes + 3 * n_axes, sys->host_axes.begin()) &&
                          sys->host_key[0] == o.r_split && sys->host_key[1] == o.band_lo &&
                          sys->host_key[2] == o.band_hi &&
                          sys->host_key[3] == batch_key(o) &&
                          sys->host_e == sys->d_f32 && sys->host_g == sys->d_g32;
        if (!same) {
            sys->drop_host_parts();
            for (int k = 0; k < parts; ++k) {
                const int nk = std::min(blk, n_axes - blk * k);
                float *ek = sys->d_f32 + blk * (size_t)k * S3;
                float *gk = sys->d_g32 + 6 * blk * (size_t)k * S3;
                vext_batch b = nullptr;
                VEXT_TRY(batch_build(1, &h, size, nk, axes + 3 * blk * k, opt, &ek, &gk, nullptr,
                                     false, &b));
                sys->host_parts.push_back(b);
                cudaEvent_t ev;
                VEXT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                sys->host_part_done.push_back(ev);
            }
            sys->host_size = size;
            sys->host_axes.assign(axes, axes + 3 * n_axes);
            sys->host_key[0] = o.r_split;
            sys->host_key[1] = o.band_lo;
            sys->host_key[2] = o.band_hi;
            sys->host_key[3] = batch_key(o);
            sys->host_e = sys->d_f32;
            sys->host_g = sys->d_g32;
        }
        for (int k = 0; k < parts; ++k) {
            const size_t first = blk * (size_t)k * S3,
                         count = std::min(blk, n_axes - blk * k) * S3;
            VEXT_TRY(batch_replay(sys->host_parts[k], st));
            VEXT_CUDA(cudaEventRecord(sys->host_part_done[k], st));
            VEXT_CUDA(cudaStreamWaitEvent(sys->aux, sys->host_part_done[k], 0));
            VEXT_CUDA(cudaMemcpyAsync(energy + first, sys->d_f32 + first, sizeof(float) * count,
                                      cudaMemcpyDeviceToHost, sys->aux));
            VEXT_CUDA(cudaMemcpyAsync(gradient + 6 * first, sys->d_g32 + 6 * first,
                                      sizeof(float) * 6 * count, cudaMemcpyDeviceToHost,
                                      sys->aux));
        }
        VEXT_CUDA(cudaStreamSynchronize(sys->aux));
        VEXT_CUDA(cudaStreamSynchronize(st));
        for (vext_batch b : sys->host_parts) VEXT_TRY(vext_batch_status(b));
        return 0;
    }
    VEXT_TRY(field_adjoint_device(h, size, n_axes, axes, o, opt, sys->d_f32, sys->d_g32, nullptr,
                                  nullptr, st));
    VEXT_CUDA(cudaMemcpyAsync(energy, sys->d_f32, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    VEXT_CUDA(cudaMemcpyAsync(gradient, sys->d_g32, sizeof(float) * 6 * n,
                              cudaMemcpyDeviceToHost, st));
    VEXT_CUDA(cudaStreamSynchronize(st));
    return check_status(sys, st);   // the FP64 modes (the mixed mode returned above)
}

extern "C" int vext_count_pairs(vext_system h, int size, int n_axes, const double *axes,
                                double r_split, int64_t *pairs, int64_t *far_pairs) {
    if (!h || !pairs || !axes || size < 1 || n_axes < 1)
        return fail(VEXT_ERR_ARGUMENT, "bad arguments");
    System *sys = &h->sys;
    std::lock_guard<std::mutex> guard(sys->lock);
    VEXT_CUDA(cudaSetDevice(sys->device));
    cudaStream_t st = sys->stream;
    vext_options d;
    vext_default_options(&d);
    d.r_split = r_split;
    const Options o = resolve_options(&d);
    RegionSet *rs = nullptr;
    // the mixed field's default region set (16 centers): far_pairs counts the
    // pairs its far kernel evaluates
    VEXT_TRY(get_field_regions(sys, size, 16, o.r_split, &rs, st));
    VEXT_TRY(ensure_capacity(sys->d_axes, sys->axes_cap, 3 * (size_t)n_axes));
    VEXT_TRY(ensure_capacity(sys->d_flags, sys->flags_cap, 4));
    VEXT_CUDA(cudaMemcpyAsync(sys->d_axes, axes, sizeof(double) * 3 * n_axes,
                              cudaMemcpyHostToDevice, st));
    unsigned long long *total = reinterpret_cast<unsigned long long *>(sys->d_flags);
    VEXT_CUDA(cudaMemsetAsync(total, 0, 2 * sizeof(unsigned long long), st));
    const FieldArgs a = make_args(sys, rs, n_axes, sys->d_axes, nullptr);
    count_kernel<<<2368, 256, 0, st>>>(a, total);
    VEXT_CUDA(cudaGetLastError());
    unsigned long long hcount[2] = {0, 0};
    VEXT_CUDA(cudaMemcpyAsync(hcount, total, sizeof hcount, cudaMemcpyDeviceToHost, st));
    VEXT_CUDA(cudaStreamSynchronize(st));
    *pairs = (int64_t)hcount[0];
    if (far_pairs) *far_pairs = (int64_t)hcount[1];
    return 0;
}
