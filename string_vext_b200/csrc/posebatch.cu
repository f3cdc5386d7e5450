// Forward + adjoint of many pose sets of different systems in ONE launch:
// the String paths of a batch of frameworks x guests (each path a few dozen
// images), evaluated every iteration.
//
// One to eight warps per pose (more for small batches).  The pose's center is
// wrapped into its system's cell and binned (the bin lists of system.cu, built
// at creation); the lanes stride over the bin's list: near entries in FP64
// from hi + lo with the contact floor, far entries in packed FP32x2 (the two
// sites in the two lanes; reciprocal of d^2 per pair, cubed) with per-lane
// FP32 partials flushed into FP64 every 16 entries.  The seven sums (E,
// dE/dsite for both sites) are reduced over the warp, then over the pose's
// warps in shared memory; a pose whose energy falls in the refinement band is
// recomputed entirely in FP64 by its warps.  Shell pairs whose FP32 d2 lies
// within kBorderTol of the cutoff (where the FP32 and FP64 cutoff tests may
// disagree) are taken in FP64 on the spot.  Outputs as
// vext_pose_energy_grad: E, dE/dcenter, tangent dE/dq, dE/du.  Pair term and
// forces as in pose.cu.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "pair.cuh"

namespace vext {

struct PoseBatchArgs {
    const PoseBatchSys *sys;
    const long long *offsets;   // [n_systems + 1]: poses of system k
    int n_systems;
    long long n;
    const double *centers, *quats;
    double *energy, *gc, *gq, *gu;
    double band_lo, band_hi;
    int *status;
    int wpp;                    // warps per pose (set at launch)
};

// This lane's far entries begin + lane + stride i < end of one pose, the two
// sites in the two lanes of the packed FP32x2 instructions (pose.cu's far loop):
// d = x - r_s, n1 = hardware reciprocal of d2, n3 = n1^3, e = n3 (c12 n3 - c6),
// fp = (n1 n3)(c6 - 2 c12 n3), dE/dsite += -6 fp d.  MASK = false for inner
// entries (within the cutoff of every pose of the bin: no mask, the shift
// summed once per entry into shift_sum).  FP32 partials are flushed into the
// FP64 sums every 16 entries.  MASK: a site whose FP32 d2 lies within
// kBorderTol of rc^2 -- where the FP32 test might decide the pair unlike the
// FP64 one -- leaves the FP32 sums and takes the pair in FP64
// (fp64_border_pair, from the hi + lo position and the FP64 site sd).
template <bool MASK>
__device__ __forceinline__ void far_lane_sums(const PoseBatchSys &y, long long base, int begin,
                                              int end, int lane, int stride, float2 nsx,
                                              float2 nsy, float2 nsz, const double (&sd)[2][3],
                                              double (&v)[7], double &shift_sum) {
    const int mine = end - begin > lane ? (end - begin - lane + stride - 1) / stride : 0;
#pragma unroll 1
    for (int i0 = 0; i0 < mine; i0 += 16) {
        float2 fe = make_float2(0.f, 0.f), gx = fe, gy = fe, gz = fe;
        float fs = 0.f;
        const int i1 = min(i0 + 16, mine);
        for (int i = i0; i < i1; ++i) {
            const long long k = base + begin + lane + (long long)stride * i;
            const float4 h = y.hi[k];
            const float4 tp = y.tf[__float_as_int(h.w)];   // (c12, c6, shift, floor2)
            const float2 dx = __fadd2_rn(make_float2(h.x, h.x), nsx),
                         dy = __fadd2_rn(make_float2(h.y, h.y), nsy),
                         dz = __fadd2_rn(make_float2(h.z, h.z), nsz);
            const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            float r0, r1;
            asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(d2.x));
            asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(d2.y));
            const float2 n1 = make_float2(r0, r1);
            float2 n3 = __fmul2_rn(__fmul2_rn(n1, n1), n1);
            if (MASK) {
                float2 m = make_float2(set_lt(d2.x, y.rc2f), set_lt(d2.y, y.rc2f));
                const float2 x = __fadd2_rn(d2, make_float2(-y.rc2f, -y.rc2f));
                const bool b0 = fabsf(x.x) < kBorderTol, b1 = fabsf(x.y) < kBorderTol;
                if (b0 || b1) {   // rare
                    const float4 l = y.lo[k];
                    const double ax = (double)h.x + (double)l.x, ay = (double)h.y + (double)l.y,
                                 az = (double)h.z + (double)l.z;
                    const int ty = __float_as_int(h.w);
                    if (b0) {
                        m.x = 0.f;
                        fp64_border_pair(sd[0][0], sd[0][1], sd[0][2], ax, ay, az, y.td, ty, y.rc2,
                                         v[0], v + 1);
                    }
                    if (b1) {
                        m.y = 0.f;
                        fp64_border_pair(sd[1][0], sd[1][1], sd[1][2], ax, ay, az, y.td, ty, y.rc2,
                                         v[0], v + 4);
                    }
                }
                n3 = __fmul2_rn(n3, m);
                fe = __ffma2_rn(m, make_float2(tp.z, tp.z), fe);
            } else {
                fs += tp.z;
            }
            fe = __ffma2_rn(n3, __ffma2_rn(make_float2(tp.x, tp.x), n3, make_float2(-tp.y, -tp.y)),
                            fe);
            const float2 fp =
                __fmul2_rn(__fmul2_rn(n1, n3),
                           __ffma2_rn(make_float2(-2.f * tp.x, -2.f * tp.x), n3,
                                      make_float2(tp.y, tp.y)));
            gx = __ffma2_rn(fp, dx, gx);
            gy = __ffma2_rn(fp, dy, gy);
            gz = __ffma2_rn(fp, dz, gz);
        }
        v[0] += (double)fe.x + (double)fe.y;
        if (!MASK) shift_sum += (double)fs;
        v[1] -= 6.0 * (double)gx.x;
        v[2] -= 6.0 * (double)gy.x;
        v[3] -= 6.0 * (double)gz.x;
        v[4] -= 6.0 * (double)gx.y;
        v[5] -= 6.0 * (double)gy.y;
        v[6] -= 6.0 * (double)gz.y;
    }
}

// Sums of one pose over its bin list: v = (E, dE/dsite0 [3], dE/dsite1 [3]),
// partial over the entries lane, lane + stride, ... (reduced by the caller).  FAR64 evaluates every entry in FP64
// (the FP64 mode, whose entries are all near, with the correctly rounded
// reciprocal; the re-evaluation of flagged poses, IEEE = false, with the
// hardware seed + two Newton steps, within an ulp or two of it); otherwise
// near entries in FP64 with the hardware reciprocal seed + one Newton step
// (relative error <= 2^-46) and far entries in packed FP32.
template <bool FAR64, bool IEEE = FAR64>
__device__ __forceinline__ void pose_sums(const PoseBatchSys &y, const RegionInfo &r,
                                          const double (&sd)[2][3], int lane, int stride,
                                          double (&v)[7]) {
    for (int e = lane; e < (FAR64 ? r.n_total : r.n_near); e += stride) {
        const float4 h = y.hi[r.off + e], l = y.lo[r.off + e];
        const double x = (double)h.x + (double)l.x, yy = (double)h.y + (double)l.y,
                     z = (double)h.z + (double)l.z;
        const int t = __float_as_int(h.w);
        const double c12 = y.td[4 * t], c6 = y.td[4 * t + 1], shift = y.td[4 * t + 2],
                     fl = y.td[4 * t + 3];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const double dx = sd[s][0] - x, dy = sd[s][1] - yy, dz = sd[s][2] - z;
            const double d2 = fma(dx, dx, fma(dy, dy, dz * dz));
            if (d2 >= y.rc2) continue;
            const double s2 = d2 < fl ? fl : d2;
            const double i2 = IEEE ? 1.0 / s2 : FAR64 ? rcp64_nr<2>(s2) : rcp64_nr<1>(s2);
            const double i6 = i2 * i2 * i2;
            v[0] += fma(i6, fma(c12, i6, -c6), shift);
            if (d2 > fl) {
                // dE/dsite = 2 dE/d(d2) (site - x),  dE/d(d2) = i2 i6 (3 c6 - 6 c12 i6)
                const double w = i2 * i6 * fma(-12.0 * c12, i6, 6.0 * c6);
                v[1 + 3 * s] = fma(w, dx, v[1 + 3 * s]);
                v[2 + 3 * s] = fma(w, dy, v[2 + 3 * s]);
                v[3 + 3 * s] = fma(w, dz, v[3 + 3 * s]);
            }
        }
    }
    if (FAR64) return;
    // far entries lie beyond r_split of every site: no contact floor
    const float2 nsx = make_float2(-(float)sd[0][0], -(float)sd[1][0]),
                 nsy = make_float2(-(float)sd[0][1], -(float)sd[1][1]),
                 nsz = make_float2(-(float)sd[0][2], -(float)sd[1][2]);
    double shift_sum = 0.0;
    far_lane_sums<false>(y, r.off, r.n_near, r.n_near + r.n_inner, lane, stride, nsx, nsy, nsz,
                         sd, v, shift_sum);
    far_lane_sums<true>(y, r.off, r.n_near + r.n_inner, r.n_total, lane, stride, nsx, nsy, nsz,
                        sd, v, shift_sum);
    v[0] += 2.0 * shift_sum;
}

__device__ __forceinline__ void warp_reduce7(double (&v)[7]) {
#pragma unroll
    for (int k = 0; k < 7; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
}

// a.wpp warps (1, 2, 4 or 8) share a pose, its lanes striding over the bin
// list together, so that small batches (a String path) still fill the GPU;
// the warps' sums are added in shared memory in a fixed order.  MIXED = false:
// the FP64 mode (every entry near, evaluated as in refinement).
template <bool MIXED>
__global__ void __launch_bounds__(256) pose_batch_kernel(PoseBatchArgs a) {
    __shared__ double part[8][7];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int W = a.wpp, per_cta = 8 / W, sub = warp % W;
    const long long groups = (a.n + per_cta - 1) / per_cta;
    for (long long grp = blockIdx.x; grp < groups; grp += gridDim.x) {   // uniform per CTA
        const long long p0 = grp * per_cta + warp / W;
        const bool live = p0 < a.n;
        const long long p = live ? p0 : a.n - 1;   // idle warps repeat the last pose, unwritten
        // system of pose p: offsets[k] <= p < offsets[k + 1]
        int lo = 0, hi = a.n_systems - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.offsets[mid] <= p) lo = mid;
            else hi = mid - 1;
        }
        const PoseBatchSys &y = a.sys[lo];
        const double *q = a.quats + 4 * p;
        const double nq = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        bool ok = isfinite(nq) && nq > 0;
        const double qw = ok ? q[0] / nq : 1.0, qx = ok ? q[1] / nq : 0.0,
                     qy = ok ? q[2] / nq : 0.0, qz = ok ? q[3] / nq : 0.0;
        const double u[3] = {1.0 - 2.0 * (qy * qy + qz * qz), 2.0 * (qx * qy + qw * qz),
                             2.0 * (qx * qz - qw * qy)};
        const double c0 = a.centers[3 * p], c1 = a.centers[3 * p + 1], c2 = a.centers[3 * p + 2];
        double f[3];
        int b[3];
        const int nb[3] = {y.nb0, y.nb1, y.nb2};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double w = c0 * y.Hinv.m[k] + c1 * y.Hinv.m[3 + k] + c2 * y.Hinv.m[6 + k];
            ok = ok && isfinite(w);
            w = isfinite(w) ? w - floor(w) : 0.0;
            if (w >= 1.0) w = 0.0;
            f[k] = w;
            b[k] = min(nb[k] - 1, (int)(w * nb[k]));
        }
        if (!ok && lane == 0) atomicExch(a.status, DEV_BAD_INPUT);
        const RegionInfo r = y.regs[(b[0] * y.nb1 + b[1]) * y.nb2 + b[2]];
        double cx, cy, cz;
        frac_to_cart(y.H, f[0] - r.of[0], f[1] - r.of[1], f[2] - r.of[2], cx, cy, cz);
        double sd[2][3];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const double off = s ? y.off1 : y.off0;
            sd[s][0] = cx + off * u[0];
            sd[s][1] = cy + off * u[1];
            sd[s][2] = cz + off * u[2];
        }
        double v[7] = {0, 0, 0, 0, 0, 0, 0};
        pose_sums<!MIXED>(y, r, sd, lane + 32 * sub, 32 * W, v);
        warp_reduce7(v);
        if (W > 1) {   // (W is a launch argument: uniform over the CTA)
            if (lane == 0)
#pragma unroll
                for (int k = 0; k < 7; ++k) part[warp][k] = v[k];
            __syncthreads();
            const int w0 = warp - sub;
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                double t = part[w0][k];
                for (int j = 1; j < W; ++j) t += part[w0 + j][k];
                v[k] = t;
            }
            __syncthreads();
        }
        // the refinement band: the pose again in FP64, by all of its warps
        // (uniform over them: each holds the pose's v[0])
        if (MIXED) {
            const bool again = v[0] > a.band_lo && v[0] < a.band_hi;
            if (again) {
#pragma unroll
                for (int k = 0; k < 7; ++k) v[k] = 0.0;
                pose_sums<true, false>(y, r, sd, lane + 32 * sub, 32 * W, v);
                warp_reduce7(v);
            }
            if (W > 1) {   // every warp of the CTA passes both barriers
                if (again && lane == 0)
#pragma unroll
                    for (int k = 0; k < 7; ++k) part[warp][k] = v[k];
                __syncthreads();
                if (again) {
                    const int w0 = warp - sub;
#pragma unroll
                    for (int k = 0; k < 7; ++k) {
                        double t = part[w0][k];
                        for (int j = 1; j < W; ++j) t += part[w0 + j][k];
                        v[k] = t;
                    }
                }
                __syncthreads();
            }
        }
        if (sub != 0) continue;
        if (live && lane == 0) {
            if (a.energy) a.energy[p] = v[0];
            double gu[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (a.gc) a.gc[3 * p + k] = v[1 + k] + v[4 + k];
                gu[k] = y.off0 * v[1 + k] + y.off1 * v[4 + k];
                if (a.gu) a.gu[3 * p + k] = gu[k];
            }
            if (a.gq) {
                // dE/dq = J(q)^T dE/du, projected on the tangent space of |q| = 1
                double g[4];
                g[0] = 2 * qz * gu[1] - 2 * qy * gu[2];
                g[1] = 2 * qy * gu[1] + 2 * qz * gu[2];
                g[2] = -4 * qy * gu[0] + 2 * qx * gu[1] - 2 * qw * gu[2];
                g[3] = -4 * qz * gu[0] + 2 * qw * gu[1] + 2 * qx * gu[2];
                const double dot = g[0] * qw + g[1] * qx + g[2] * qy + g[3] * qz;
                const double inv = ok ? 1.0 / nq : 0.0;
                a.gq[4 * p + 0] = (g[0] - dot * qw) * inv;
                a.gq[4 * p + 1] = (g[1] - dot * qx) * inv;
                a.gq[4 * p + 2] = (g[2] - dot * qy) * inv;
                a.gq[4 * p + 3] = (g[3] - dot * qz) * inv;
            }
        }
    }
}

// Warps per pose: the smallest power of two up to 8 that gives about 16
// resident warps per SM (148 SMs), so small batches spread each pose's list
// over several warps.
static int warps_per_pose(long long n) {
    int w = 1;
    while (w < 8 && n * (2 * w) <= 148LL * 16) w *= 2;
    return w;
}

static int pose_batch_launch(PoseBatchArgs a, bool mixed, cudaStream_t st) {
    a.wpp = warps_per_pose(a.n);
    const long long groups = (a.n + 8 / a.wpp - 1) / (8 / a.wpp);
    const int blocks = (int)std::min<long long>(groups, 148LL * 16);
    if (mixed) pose_batch_kernel<true><<<blocks, 256, 0, st>>>(a);
    else pose_batch_kernel<false><<<blocks, 256, 0, st>>>(a);
    VEXT_CUDA(cudaGetLastError());
    return 0;
}

static PoseBatchSys describe(const System *sys, const RegionSet *rs) {
    PoseBatchSys y;
    std::memset(&y, 0, sizeof y);   // padding too: descriptors are compared bytewise
    y.H = sys->H;
    y.Hinv = sys->Hinv;
    y.rc2 = sys->cutoff * sys->cutoff;
    y.rc2f = (float)y.rc2;
    y.off0 = sys->offsets[0];
    y.off1 = sys->offsets[1];
    y.nb0 = rs->nb[0];
    y.nb1 = rs->nb[1];
    y.nb2 = rs->nb[2];
    y.regs = rs->d_info;
    y.hi = rs->d_hi;
    y.lo = rs->d_lo;
    y.td = sys->d_td;
    y.tf = sys->d_tf;
    return y;
}

int pose_warp_enqueue(System *sys, const RegionSet *rs, int n, const double *centers,
                      const double *quats, const Options &o, double *energy, double *gc,
                      double *gq, double *gu, cudaStream_t st) {
    // The descriptor is uploaded synchronously on first use and whenever the
    // bin lists moved (compared with the host copy of the last upload); inside
    // a stream capture it is therefore already in place.
    const PoseBatchSys y = describe(sys, rs);
    const bool upload =
        !sys->d_pose_desc || std::memcmp(&sys->h_pose_desc, &y, sizeof y) != 0;
    if (!sys->d_pose_desc) {
        VEXT_CUDA(cudaMalloc(&sys->d_pose_desc, sizeof(PoseBatchSys)));
        VEXT_CUDA(cudaMalloc(&sys->d_pose_offsets, 2 * sizeof(long long)));
        const long long off[2] = {0, 0};   // one system: the kernel never reads them
        VEXT_CUDA(cudaMemcpy(sys->d_pose_offsets, off, sizeof off, cudaMemcpyHostToDevice));
    }
    if (upload) {
        VEXT_CUDA(cudaMemcpy(sys->d_pose_desc, &y, sizeof y, cudaMemcpyHostToDevice));
        std::memcpy(&sys->h_pose_desc, &y, sizeof y);
    }
    PoseBatchArgs a;
    a.sys = sys->d_pose_desc;
    a.offsets = sys->d_pose_offsets;
    a.n_systems = 1;
    a.n = n;
    a.centers = centers;
    a.quats = quats;
    a.energy = energy;
    a.gc = gc;
    a.gq = gq;
    a.gu = gu;
    const bool band = o.mode == VEXT_MODE_MIXED && o.band_hi > o.band_lo;
    a.band_lo = band ? o.band_lo : 0.0;
    a.band_hi = band ? o.band_hi : 0.0;
    a.status = sys->d_status;
    return pose_batch_launch(a, o.mode == VEXT_MODE_MIXED, st);
}

}  // namespace vext

using namespace vext;

struct vext_pose_batch_s {
    std::vector<vext_system> systems;
    long long n = 0;
    int n_systems = 0;
    Options opt;
    PoseBatchSys *d_sys = nullptr;
    long long *d_offsets = nullptr;
    int *d_status = nullptr;
    ~vext_pose_batch_s() {
        cudaFree(d_sys);
        cudaFree(d_offsets);
        cudaFree(d_status);
    }
};

extern "C" int vext_pose_batch_create(int n_systems, const vext_system *systems,
                                      const int64_t *pose_offsets, const vext_options *opt,
                                      vext_pose_batch *out) {
    if (!out || n_systems < 1 || !systems || !pose_offsets)
        return fail(VEXT_ERR_ARGUMENT, "bad pose batch arguments");
    *out = nullptr;
    if (pose_offsets[0] != 0) return fail(VEXT_ERR_ARGUMENT, "pose_offsets[0] must be 0");
    for (int k = 0; k < n_systems; ++k) {
        if (!systems[k]) return fail(VEXT_ERR_ARGUMENT, "null system %d", k);
        if (pose_offsets[k + 1] < pose_offsets[k])
            return fail(VEXT_ERR_ARGUMENT, "pose_offsets must not decrease");
    }
    auto *b = new vext_pose_batch_s();
    std::unique_ptr<vext_pose_batch_s> guard(b);
    b->systems.assign(systems, systems + n_systems);
    b->n_systems = n_systems;
    b->n = pose_offsets[n_systems];
    b->opt = resolve_options(opt);
    if (b->opt.mode != VEXT_MODE_MIXED && b->opt.mode != VEXT_MODE_FP64)
        return fail(VEXT_ERR_ARGUMENT, "unknown precision mode %d", b->opt.mode);
    const double r_split = b->opt.mode == VEXT_MODE_FP64 ? 1e30 : b->opt.r_split;
    int dev = 0;
    VEXT_CUDA(cudaGetDevice(&dev));
    std::vector<PoseBatchSys> hs(n_systems);
    for (int k = 0; k < n_systems; ++k) {
        System *sys = &systems[k]->sys;
        if (sys->device != dev)
            return fail(VEXT_ERR_ARGUMENT, "system %d lives on another device", k);
        std::lock_guard<std::mutex> lock(sys->lock);
        RegionSet *rs = nullptr;
        VEXT_TRY(get_bin_regions(sys, r_split, &rs, sys->stream));
        hs[k] = describe(sys, rs);
    }
    std::vector<long long> offs(pose_offsets, pose_offsets + n_systems + 1);
    VEXT_CUDA(cudaMalloc(&b->d_sys, sizeof(PoseBatchSys) * n_systems));
    VEXT_CUDA(cudaMemcpy(b->d_sys, hs.data(), sizeof(PoseBatchSys) * n_systems,
                         cudaMemcpyHostToDevice));
    VEXT_CUDA(cudaMalloc(&b->d_offsets, sizeof(long long) * (n_systems + 1)));
    VEXT_CUDA(cudaMemcpy(b->d_offsets, offs.data(), sizeof(long long) * (n_systems + 1),
                         cudaMemcpyHostToDevice));
    VEXT_CUDA(cudaMalloc(&b->d_status, sizeof(int)));
    VEXT_CUDA(cudaMemset(b->d_status, 0, sizeof(int)));
    *out = guard.release();
    return 0;
}

extern "C" int vext_pose_batch_run(vext_pose_batch b, const double *centers, const double *quats,
                                   double *energy, double *grad_center, double *grad_quat,
                                   double *grad_director, void *stream) {
    if (!b) return fail(VEXT_ERR_ARGUMENT, "null pose batch");
    if (b->n == 0) return 0;
    if (!centers || !quats) return fail(VEXT_ERR_ARGUMENT, "centers and quaternions required");
    PoseBatchArgs a;
    a.sys = b->d_sys;
    a.offsets = b->d_offsets;
    a.n_systems = b->n_systems;
    a.n = b->n;
    a.centers = centers;
    a.quats = quats;
    a.energy = energy;
    a.gc = grad_center;
    a.gq = grad_quat;
    a.gu = grad_director;
    const bool band = b->opt.mode == VEXT_MODE_MIXED && b->opt.band_hi > b->opt.band_lo;
    a.band_lo = band ? b->opt.band_lo : 0.0;
    a.band_hi = band ? b->opt.band_hi : 0.0;
    a.status = b->d_status;
    return pose_batch_launch(a, b->opt.mode == VEXT_MODE_MIXED, (cudaStream_t)stream);
}

extern "C" int vext_pose_batch_status(vext_pose_batch b) {
    if (!b) return fail(VEXT_ERR_ARGUMENT, "null pose batch");
    int h = 0;
    VEXT_CUDA(cudaDeviceSynchronize());
    VEXT_CUDA(cudaMemcpy(&h, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        VEXT_CUDA(cudaMemset(b->d_status, 0, sizeof(int)));
        if (h == DEV_BAD_INPUT) return fail(VEXT_ERR_ARGUMENT, "non-finite pose center or zero quaternion");
        return fail(VEXT_ERR_TIMEOUT, "device status %d", h);
    }
    return 0;
}

extern "C" int vext_pose_batch_destroy(vext_pose_batch b) {
    delete b;
    return 0;
}
