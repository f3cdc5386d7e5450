// Systems (framework + guest resident on the device) and their region lists.
//
// The pair coefficients follow the reference's ReusePotential
// (src/string_vext/neighbor.py:21-28) in FP64: sigma = (sigma_f + sigma_g)/2,
// eps = sqrt(eps_f eps_g), c12 = 4 eps sigma^12, c6 = 4 eps sigma^6,
// shift = -4 eps ((sigma/rc)^12 - (sigma/rc)^6), floor2 = (0.1 sigma)^2.
//
// Image enumeration (replacing TriclinicSitePotential's fixed reach box and
// kd-tree, physics.py:43-57): for a region with fractional origin f_o and
// radius rho, every (atom j, lattice shift n) whose image lies within
// R = rc + max|offset| + rho of the origin is listed.  Along axis k the
// fractional extent of a ball of radius R is R |Hinv[:,k]|, so n_k runs over
// [ceil(-d_k - R e_k), floor(-d_k + R e_k)] with d = f_j - f_o; the exact
// distance test is done in FP64 on (d + n) @ H.  No minimum image is used.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

#include "internal.cuh"

namespace vext {

// ------------------------------------------------------------ error state

static thread_local std::string g_error;

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
}

int fail(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

Options resolve_options(const vext_options *opt) {
    vext_options d;
    vext_default_options(&d);
    if (!opt) opt = &d;
    Options o;
    o.mode = opt->mode;
    // Far pairs skip the contact floor, so r_split must exceed every floor
    // distance 0.1 sigma: it is clamped to at least 1 A.
    o.r_split = opt->r_split > 0 ? std::max(opt->r_split, 1.0) : kDefaultRSplit;
    o.band_lo = opt->band_lo;
    o.band_hi = opt->band_hi;
    o.cb = opt->centers_per_region;
    o.variant = opt->variant;
    o.batch_shape = opt->batch_shape;
    return o;
}

// ------------------------------------------------------------ block shapes

double block_radius(const Mat3 &H, int size, int ni, int nj, int nk) {
    // Centers of one block span (n-1)/S along each fractional axis; the
    // farthest center from the block's mean is a corner of that box.
    const double ha = 0.5 * (ni - 1) / size, hb = 0.5 * (nj - 1) / size,
                 hc = 0.5 * (nk - 1) / size;
    double best = 0;
    for (int s = 0; s < 8; ++s) {
        double x, y, z;
        frac_to_cart(H, (s & 1 ? ha : -ha), (s & 2 ? hb : -hb), (s & 4 ? hc : -hc), x, y, z);
        best = std::max(best, std::sqrt(x * x + y * y + z * z));
    }
    return best;
}

void choose_block_shape(const Mat3 &H, int size, int cb, int &bi, int &bj, int &bk) {
    double best = 1e300;
    bi = bj = 1;
    bk = std::min(cb, size);
    for (int a = 1; a <= cb; ++a)
        for (int b = 1; a * b <= cb; ++b) {
            if (cb % (a * b)) continue;
            const int c = cb / (a * b);
            if (a > size || b > size || c > size) continue;
            const double r = block_radius(H, size, a, b, c);
            if (r < best - 1e-12) {
                best = r;
                bi = a;
                bj = b;
                bk = c;
            }
        }
}

// ------------------------------------------------------------ list build

struct BuildArgs {
    Mat3 H;
    double einv[3];
    const double *frac;
    const int *type;
    int n_atoms;
    double r_list0;   // rc + max|offset| (+ margin)
    double r_near0;   // r_split + max|offset| (+ margin)
    double r_inner0;  // cutoff - max|offset| (- margin): inner entries lie within r_inner0 - rho
    double r_outer0;  // cutoff + 1e-3 A: outer shell entries lie beyond r_outer0 + rho
};

// Visit every candidate image of atom j for a region; f(dist2, rel) per image.
template <typename F>
__device__ __forceinline__ void for_each_image(const BuildArgs &a, const RegionInfo &r, int j,
                                               double rl, F &&f) {
    const double d0 = a.frac[3 * j] - r.of[0];
    const double d1 = a.frac[3 * j + 1] - r.of[1];
    const double d2 = a.frac[3 * j + 2] - r.of[2];
    const double e0 = __dmul_rn(rl, a.einv[0]), e1 = __dmul_rn(rl, a.einv[1]),
                 e2 = __dmul_rn(rl, a.einv[2]);
    const int lo0 = (int)ceil(__dsub_rn(-d0, e0)), hi0 = (int)floor(__dadd_rn(-d0, e0));
    const int lo1 = (int)ceil(__dsub_rn(-d1, e1)), hi1 = (int)floor(__dadd_rn(-d1, e1));
    const int lo2 = (int)ceil(__dsub_rn(-d2, e2)), hi2 = (int)floor(__dadd_rn(-d2, e2));
    const double rl2 = rl * rl;
    for (int n0 = lo0; n0 <= hi0; ++n0)
        for (int n1 = lo1; n1 <= hi1; ++n1)
            for (int n2 = lo2; n2 <= hi2; ++n2) {
                // explicit FMAs: the count and fill kernels must take
                // bit-identical decisions for every candidate
                const double u = d0 + n0, v = d1 + n1, w = d2 + n2;
                const double x = fma(u, a.H.m[0], fma(v, a.H.m[3], __dmul_rn(w, a.H.m[6])));
                const double y = fma(u, a.H.m[1], fma(v, a.H.m[4], __dmul_rn(w, a.H.m[7])));
                const double z = fma(u, a.H.m[2], fma(v, a.H.m[5], __dmul_rn(w, a.H.m[8])));
                const double q = fma(x, x, fma(y, y, __dmul_rn(z, z)));
                if (q < rl2) f(q, x, y, z);
            }
}

template <int NT>
__device__ __forceinline__ void block_scan2(int a, int b, int &pa, int &pb, int &ta, int &tb,
                                            int *sh) {
    // Exclusive scan of two ints over the block (NT threads, NT <= 1024).
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int xa = a, xb = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int ya = __shfl_up_sync(0xffffffffu, xa, o);
        const int yb = __shfl_up_sync(0xffffffffu, xb, o);
        if (lane >= o) {
            xa += ya;
            xb += yb;
        }
    }
    if (lane == 31) {
        sh[warp] = xa;
        sh[32 + warp] = xb;
    }
    __syncthreads();
    if (warp == 0) {
        int va = lane < NT / 32 ? sh[lane] : 0, vb = lane < NT / 32 ? sh[32 + lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int ya = __shfl_up_sync(0xffffffffu, va, o);
            const int yb = __shfl_up_sync(0xffffffffu, vb, o);
            if (lane >= o) {
                va += ya;
                vb += yb;
            }
        }
        sh[64 + lane] = va;   // inclusive warp prefixes
        sh[96 + lane] = vb;
    }
    __syncthreads();
    const int wa = warp ? sh[64 + warp - 1] : 0, wb = warp ? sh[96 + warp - 1] : 0;
    pa = wa + xa - a;
    pb = wb + xb - b;
    ta = sh[64 + NT / 32 - 1];
    tb = sh[96 + NT / 32 - 1];
    __syncthreads();
}

constexpr int kBuildThreads = 256;

// Per region: the entries of each class, and per thread (atoms j = tid, tid +
// kBuildThreads, ...) its (near, inner, shell, outer) counts for the fill.
__global__ void __launch_bounds__(kBuildThreads)
    region_count_kernel(BuildArgs a, RegionInfo *regs, int n_regions, int4 *counts) {
    const int region = blockIdx.x;
    if (region >= n_regions) return;
    const RegionInfo r = regs[region];
    const double rl = a.r_list0 + r.rho, rn = a.r_near0 + r.rho, rn2 = rn * rn;
    const double ri = a.r_inner0 - r.rho, ri2 = ri > 0 ? ri * ri : 0.0;
    const double ro = a.r_outer0 + r.rho, ro2 = ro * ro;
    int near = 0, inner = 0, outer = 0, total = 0;
    for (int j = threadIdx.x; j < a.n_atoms; j += kBuildThreads)
        for_each_image(a, r, j, rl, [&](double q, double, double, double) {
            ++total;
            near += q < rn2;
            inner += q >= rn2 && q < ri2;
            outer += q >= rn2 && q >= ri2 && q >= ro2;
        });
    counts[(long long)region * kBuildThreads + threadIdx.x] =
        make_int4(near, inner, total - near - inner - outer, outer);
    __shared__ int sh[128];
    int pa, pb, ta, tb, pc, pd, tc, td;
    block_scan2<kBuildThreads>(near, total, pa, pb, ta, tb, sh);
    block_scan2<kBuildThreads>(inner, outer, pc, pd, tc, td, sh);
    if (threadIdx.x == 0) {
        regs[region].n_near = ta;
        regs[region].n_total = tb;
        regs[region].n_inner = tc;
        regs[region].n_outer = td;
    }
}

// Entry order inside each class: thread-major (thread t's atoms t, t +
// kBuildThreads, ... in turn, each atom's images in enumeration order), so a
// thread's slots follow from a block scan of the per-thread counts that
// region_count_kernel stored and the candidates are enumerated once here.
__global__ void __launch_bounds__(kBuildThreads, 2)
    region_fill_kernel(BuildArgs a, const RegionInfo *regs, int n_regions, const int4 *counts,
                       float4 *hi, float4 *lo, int *status) {
    const int region = blockIdx.x;
    if (region >= n_regions) return;
    const RegionInfo r = regs[region];
    const double rl = a.r_list0 + r.rho, rn = a.r_near0 + r.rho, rn2 = rn * rn;
    const double ri = a.r_inner0 - r.rho, ri2 = ri > 0 ? ri * ri : 0.0;
    const double ro = a.r_outer0 + r.rho, ro2 = ro * ro;
    __shared__ int sh[128];
    // entry order: near | far inner | far shell | outer shell
    const int end_shell = r.n_total - r.n_outer;
    const int4 c = counts[(long long)region * kBuildThreads + threadIdx.x];
    int pn, pi, tn, ti, ps, po, ts, to;
    block_scan2<kBuildThreads>(c.x, c.y, pn, pi, tn, ti, sh);
    block_scan2<kBuildThreads>(c.z, c.w, ps, po, ts, to, sh);
    if (threadIdx.x == 0 && (tn != r.n_near || ti != r.n_inner ||
                             ts != end_shell - r.n_near - r.n_inner || to != r.n_outer))
        atomicExch(status, DEV_BAD_LIST);
    // this thread's next slot and end per class (scalars: an indexed array
    // would live in local memory)
    int wn = pn, wi = r.n_near + pi, ws = r.n_near + r.n_inner + ps, wo = end_shell + po;
    const int en = wn + c.x, ei = wi + c.y, es = ws + c.z, eo = wo + c.w;
    for (int j = threadIdx.x; j < a.n_atoms; j += kBuildThreads) {
        const int t = a.type[j];
        for_each_image(a, r, j, rl, [&](double q, double x, double y, double z) {
            const int cls = q < rn2 ? 0 : (q < ri2 ? 1 : (q < ro2 ? 2 : 3));
            const int slot = cls == 0 ? wn++ : (cls == 1 ? wi++ : (cls == 2 ? ws++ : wo++));
            const int lim = cls == 0 ? en : (cls == 1 ? ei : (cls == 2 ? es : eo));
            if (slot >= lim) {
                atomicExch(status, DEV_BAD_LIST);
                return;
            }
            const float hx = (float)x, hy = (float)y, hz = (float)z;
            hi[r.off + slot] = make_float4(hx, hy, hz, __int_as_float(t));
            lo[r.off + slot] = make_float4((float)(x - hx), (float)(y - hy), (float)(z - hz), 0.f);
        });
    }
    if (wn != en || wi != ei || ws != es || wo != eo) atomicExch(status, DEV_BAD_LIST);
}

// ------------------------------------------------------------ region sets

RegionSet::~RegionSet() {
    cudaFree(d_info);
    cudaFree(d_hi);
    cudaFree(d_lo);
}

// Per-device scratch of the per-(region, thread) class counts that the count
// pass hands to the fill pass; one list build at a time uses it (the lock is
// held until the build's kernels have finished).  It belongs to the context
// it was allocated in: after a device reset (a new context, told apart by
// its unique id) the old array is gone and a new one is allocated.
namespace {
struct BuildScratch {
    std::mutex lock;
    int4 *ptr = nullptr;
    size_t cap = 0;
    unsigned long long ctx_id = 0;
};
// Unique id of the calling thread's current context (0 when unavailable).
unsigned long long current_context_id() {
    using GetCurrentFn = CUresult (*)(CUcontext *);
    using GetIdFn = CUresult (*)(CUcontext, unsigned long long *);
    static const std::pair<GetCurrentFn, GetIdFn> fns = [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa = cudaDriverEntryPointSymbolNotFound, qb = qa;
        const bool ok =
            cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) ==
                cudaSuccess &&
            qa == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess;
        if (!ok) {
            cudaGetLastError();
            return std::pair<GetCurrentFn, GetIdFn>(nullptr, nullptr);
        }
        return std::pair<GetCurrentFn, GetIdFn>(reinterpret_cast<GetCurrentFn>(a),
                                                reinterpret_cast<GetIdFn>(b));
    }();
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!fns.first || fns.first(&ctx) != CUDA_SUCCESS || !ctx || fns.second(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}
BuildScratch &build_scratch(int device) {
    static BuildScratch scratch[64];
    return scratch[device & 63];
}
// Waits for the stream before the scratch lock is released, also on the
// early error returns of build_lists.
struct StreamDrain {
    cudaStream_t stream;
    ~StreamDrain() { cudaStreamSynchronize(stream); }
};
}  // namespace

static int build_lists(System *sys, RegionSet *rs, cudaStream_t stream) {
    BuildScratch &scratch = build_scratch(sys->device);
    std::lock_guard<std::mutex> scratch_guard(scratch.lock);
    StreamDrain drain{stream};
    BuildArgs a;
    a.H = sys->H;
    for (int k = 0; k < 3; ++k) a.einv[k] = sys->einv[k];
    a.frac = sys->d_frac;
    a.type = sys->d_type;
    a.n_atoms = sys->n_atoms;
    // 1e-6 A margins keep every pair within rc (resp. r_split) listed despite
    // FP64 rounding of the distances (~1e-14 A).
    a.r_list0 = sys->cutoff + sys->max_offset + 1e-6;
    a.r_near0 = rs->r_split + sys->max_offset + 1e-6;
    a.r_inner0 = sys->cutoff - sys->max_offset - 1e-6;
    a.r_outer0 = sys->cutoff + 1e-3;
    const int n = rs->n_regions;
    if (!rs->d_info) VEXT_CUDA(cudaMalloc(&rs->d_info, sizeof(RegionInfo) * n));
    VEXT_CUDA(cudaMemcpyAsync(rs->d_info, rs->h_info.data(), sizeof(RegionInfo) * n,
                              cudaMemcpyHostToDevice, stream));
    cudaEvent_t e0 = sys->ev[3], e1 = sys->ev[4];
    VEXT_CUDA(cudaEventRecord(e0, stream));
    const unsigned long long ctx = current_context_id();
    if (scratch.ptr && ctx != 0 && scratch.ctx_id != 0 && ctx != scratch.ctx_id) {
        // allocated in a context that has since been reset: it went with that
        // context; allocate anew
        scratch.ptr = nullptr;
        scratch.cap = 0;
    }
    VEXT_TRY(ensure_capacity(scratch.ptr, scratch.cap, (size_t)n * kBuildThreads));
    scratch.ctx_id = ctx;
    region_count_kernel<<<n, kBuildThreads, 0, stream>>>(a, rs->d_info, n, scratch.ptr);
    VEXT_CUDA(cudaGetLastError());
    VEXT_CUDA(cudaMemcpyAsync(rs->h_info.data(), rs->d_info, sizeof(RegionInfo) * n,
                              cudaMemcpyDeviceToHost, stream));
    VEXT_CUDA(cudaStreamSynchronize(stream));
    long long off = 0, near = 0, outer = 0;
    for (auto &r : rs->h_info) {
        r.off = off;
        off += r.n_total;
        near += r.n_near;
        outer += r.n_outer;
    }
    rs->n_entries = off;
    rs->n_near = near;
    rs->n_outer = outer;
    VEXT_CUDA(cudaMemcpyAsync(rs->d_info, rs->h_info.data(), sizeof(RegionInfo) * n,
                              cudaMemcpyHostToDevice, stream));
    if (off > rs->capacity || !rs->d_hi) {
        cudaFree(rs->d_hi);
        cudaFree(rs->d_lo);
        rs->d_hi = rs->d_lo = nullptr;
        rs->capacity = 0;
        VEXT_CUDA(cudaMalloc(&rs->d_hi, sizeof(float4) * std::max<long long>(off, 1)));
        VEXT_CUDA(cudaMalloc(&rs->d_lo, sizeof(float4) * std::max<long long>(off, 1)));
        rs->capacity = std::max<long long>(off, 1);
    }
    region_fill_kernel<<<n, kBuildThreads, 0, stream>>>(a, rs->d_info, n, scratch.ptr, rs->d_hi,
                                                        rs->d_lo, sys->d_status);
    VEXT_CUDA(cudaGetLastError());
    VEXT_CUDA(cudaEventRecord(e1, stream));
    VEXT_CUDA(cudaEventSynchronize(e1));
    VEXT_CUDA(cudaEventElapsedTime(&rs->build_ms, e0, e1));
    sys->list_timed = true;
    rs->stale = false;
    return check_status(sys, stream);
}

int get_field_regions(System *sys, int size, int cb, double r_split, RegionSet **out,
                      cudaStream_t stream) {
    for (RegionSet *rs : sys->sets)
        if (rs->size == size && rs->bi * rs->bj * rs->bk == cb && rs->r_split == r_split) {
            if (rs->stale) {
                for (auto &r : rs->h_info) r.n_near = r.n_total = r.n_inner = r.n_outer = 0;
                VEXT_TRY(build_lists(sys, rs, stream));
            }
            *out = rs;
            return 0;
        }
    RegionSet *rs = new RegionSet();
    rs->size = size;
    rs->r_split = r_split;
    choose_block_shape(sys->H, size, cb, rs->bi, rs->bj, rs->bk);
    rs->n_ri = (size + rs->bi - 1) / rs->bi;
    rs->n_rj = (size + rs->bj - 1) / rs->bj;
    rs->n_rk = (size + rs->bk - 1) / rs->bk;
    rs->n_regions = rs->n_ri * rs->n_rj * rs->n_rk;
    rs->h_info.resize(rs->n_regions);
    int idx = 0;
    for (int I = 0; I < rs->n_ri; ++I)
        for (int J = 0; J < rs->n_rj; ++J)
            for (int K = 0; K < rs->n_rk; ++K) {
                RegionInfo &r = rs->h_info[idx++];
                std::memset(&r, 0, sizeof r);
                r.i0 = I * rs->bi;
                r.j0 = J * rs->bj;
                r.k0 = K * rs->bk;
                r.ni = std::min(rs->bi, size - r.i0);
                r.nj = std::min(rs->bj, size - r.j0);
                r.nk = std::min(rs->bk, size - r.k0);
                // origin = mean of the block's centers ((i + .5)/S ...)
                r.of[0] = (r.i0 + 0.5 * r.ni) / size;
                r.of[1] = (r.j0 + 0.5 * r.nj) / size;
                r.of[2] = (r.k0 + 0.5 * r.nk) / size;
                r.rho = block_radius(sys->H, size, r.ni, r.nj, r.nk) + 1e-9;
            }
    int rc = build_lists(sys, rs, stream);
    if (rc) {
        delete rs;
        return rc;
    }
    sys->sets.push_back(rs);
    *out = rs;
    return 0;
}

// Width (A, between lattice planes) of the pose bins.

int get_bin_regions(System *sys, double r_split, RegionSet **out, cudaStream_t stream,
                    double bin_width) {
    for (RegionSet *rs : sys->sets)
        if (rs->size == 0 && rs->r_split == r_split && rs->bin_width == bin_width) {
            if (rs->stale) {
                for (auto &r : rs->h_info) r.n_near = r.n_total = r.n_inner = r.n_outer = 0;
                VEXT_TRY(build_lists(sys, rs, stream));
            }
            *out = rs;
            return 0;
        }
    RegionSet *rs = new RegionSet();
    rs->r_split = r_split;
    rs->bin_width = bin_width;
    // Bins about bin_width wide between lattice planes.
    for (int k = 0; k < 3; ++k)
        rs->nb[k] = std::max(1, (int)std::ceil((1.0 / sys->einv[k]) / bin_width));
    rs->n_ri = rs->nb[0];
    rs->n_rj = rs->nb[1];
    rs->n_rk = rs->nb[2];
    rs->n_regions = rs->nb[0] * rs->nb[1] * rs->nb[2];
    rs->h_info.resize(rs->n_regions);
    int idx = 0;
    for (int I = 0; I < rs->nb[0]; ++I)
        for (int J = 0; J < rs->nb[1]; ++J)
            for (int K = 0; K < rs->nb[2]; ++K) {
                RegionInfo &r = rs->h_info[idx++];
                std::memset(&r, 0, sizeof r);
                r.of[0] = (I + 0.5) / rs->nb[0];
                r.of[1] = (J + 0.5) / rs->nb[1];
                r.of[2] = (K + 0.5) / rs->nb[2];
                // half-diagonal of the bin parallelepiped (any wrapped center
                // in the bin, boundaries included)
                double best = 0;
                for (int s = 0; s < 8; ++s) {
                    double x, y, z;
                    frac_to_cart(sys->H, (s & 1 ? 0.5 : -0.5) / rs->nb[0],
                                 (s & 2 ? 0.5 : -0.5) / rs->nb[1], (s & 4 ? 0.5 : -0.5) / rs->nb[2],
                                 x, y, z);
                    best = std::max(best, std::sqrt(x * x + y * y + z * z));
                }
                r.rho = best + 1e-9;
            }
    int rc = build_lists(sys, rs, stream);
    if (rc) {
        delete rs;
        return rc;
    }
    sys->sets.push_back(rs);
    *out = rs;
    return 0;
}

int check_status(System *sys, cudaStream_t stream) {
    int h = 0;
    VEXT_CUDA(cudaMemcpyAsync(&h, sys->d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    VEXT_CUDA(cudaStreamSynchronize(stream));
    if (h == DEV_OK) return 0;
    VEXT_CUDA(cudaMemsetAsync(sys->d_status, 0, sizeof(int), stream));
    VEXT_CUDA(cudaStreamSynchronize(stream));
    if (h == DEV_TIMEOUT) return fail(VEXT_ERR_TIMEOUT, "a device wait gave up (status %d)", h);
    return fail(VEXT_ERR_CUDA, "device list build inconsistency (status %d)", h);
}

void System::drop_adjoint_batch() {
    if (adj_batch) vext_batch_destroy(adj_batch);
    adj_batch = nullptr;
    adj_size = 0;
    adj_axes.clear();
    drop_host_parts();
}

void System::drop_host_parts() {
    for (vext_batch b : host_parts) vext_batch_destroy(b);
    for (cudaEvent_t e : host_part_done) cudaEventDestroy(e);
    host_parts.clear();
    host_part_done.clear();
    host_size = 0;
    host_axes.clear();
}

System::~System() {
    drop_adjoint_batch();   // it points into the region sets
    for (RegionSet *rs : sets) delete rs;
    cudaFree(d_g32);
    cudaFree(d_frac);
    cudaFree(d_type);
    cudaFree(d_tf);
    cudaFree(d_td);
    cudaFree(d_status);
    cudaFree(d_e64);
    cudaFree(d_refine);
    cudaFree(d_axes);
    cudaFree(d_f32);
    cudaFree(d_small);
    cudaFree(d_e64T);
    cudaFree(d_flags);
    cudaFree(d_pose_scratch);
    cudaFree(d_pose_io);
    cudaFree(d_pose_desc);
    cudaFree(d_pose_offsets);
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (aux) cudaStreamDestroy(aux);
    if (stream) cudaStreamDestroy(stream);
}

}  // namespace vext

using namespace vext;

extern "C" void vext_default_options(vext_options *opt) {
    std::memset(opt, 0, sizeof *opt);
    opt->mode = VEXT_MODE_MIXED;
    opt->r_split = kDefaultRSplit;
    opt->band_lo = -1e-2;
    opt->band_hi = 100.0;
    opt->centers_per_region = 0;
}

extern "C" const char *vext_last_error(void) { return g_error.c_str(); }

extern "C" const char *vext_version(void) { return "vext_b200 0.1.0 (sm_100a)"; }

extern "C" int vext_system_create(const vext_system_desc *d, vext_system *out) {
    if (!d || !out) return fail(VEXT_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    if (d->n_atoms < 1 || !d->frac || !d->sigma || !d->epsilon)
        return fail(VEXT_ERR_ARGUMENT, "at least one framework atom with sigma/epsilon required");
    if (!(d->cutoff > 0) || !std::isfinite(d->cutoff))
        return fail(VEXT_ERR_ARGUMENT, "positive finite cutoff required");
    if (!(d->guest_sigma > 0) || !(d->guest_epsilon > 0))
        return fail(VEXT_ERR_ARGUMENT, "positive guest sigma/epsilon required");
    if (!std::isfinite(d->offsets[0]) || !std::isfinite(d->offsets[1]))
        return fail(VEXT_ERR_ARGUMENT, "finite site offsets required");
    const double *h = d->cell;
    for (int k = 0; k < 9; ++k)
        if (!std::isfinite(h[k])) return fail(VEXT_ERR_ARGUMENT, "non-finite cell");
    const double det = h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
                       h[2] * (h[3] * h[7] - h[4] * h[6]);
    if (!(det > 0)) return fail(VEXT_ERR_ARGUMENT, "cell determinant must be positive");
    for (int i = 0; i < d->n_atoms; ++i) {
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(d->frac[3 * i + k]))
                return fail(VEXT_ERR_ARGUMENT, "non-finite fractional coordinate (atom %d)", i);
        if (!(d->sigma[i] > 0) || !(d->epsilon[i] > 0) || !std::isfinite(d->sigma[i]) ||
            !std::isfinite(d->epsilon[i]))
            return fail(VEXT_ERR_ARGUMENT, "invalid framework LJ parameters (atom %d)", i);
    }
    auto *handle = new vext_system_s();
    System &s = handle->sys;
    cudaGetDevice(&s.device);
    std::memcpy(s.H.m, h, sizeof s.H.m);
    // inverse via the adjugate
    const double *m = h;
    double inv[9] = {(m[4] * m[8] - m[5] * m[7]) / det, (m[2] * m[7] - m[1] * m[8]) / det,
                     (m[1] * m[5] - m[2] * m[4]) / det, (m[5] * m[6] - m[3] * m[8]) / det,
                     (m[0] * m[8] - m[2] * m[6]) / det, (m[2] * m[3] - m[0] * m[5]) / det,
                     (m[3] * m[7] - m[4] * m[6]) / det, (m[1] * m[6] - m[0] * m[7]) / det,
                     (m[0] * m[4] - m[1] * m[3]) / det};
    std::memcpy(s.Hinv.m, inv, sizeof inv);
    for (int k = 0; k < 3; ++k)
        s.einv[k] = std::sqrt(inv[k] * inv[k] + inv[3 + k] * inv[3 + k] + inv[6 + k] * inv[6 + k]);
    s.n_atoms = d->n_atoms;
    s.guest_sigma = d->guest_sigma;
    s.guest_epsilon = d->guest_epsilon;
    s.offsets[0] = d->offsets[0];
    s.offsets[1] = d->offsets[1];
    s.max_offset = std::max(std::fabs(d->offsets[0]), std::fabs(d->offsets[1]));
    s.cutoff = d->cutoff;
    s.temperature = d->temperature;
    // distinct (sigma, epsilon) pairs -> type ids, in order of first appearance
    std::map<std::pair<double, double>, int> ids;
    std::vector<int> type(d->n_atoms);
    std::vector<double> frac(3 * (size_t)d->n_atoms);
    for (int i = 0; i < d->n_atoms; ++i) {
        auto key = std::make_pair(d->sigma[i], d->epsilon[i]);
        auto it = ids.find(key);
        if (it == ids.end()) it = ids.emplace(key, (int)ids.size()).first;
        type[i] = it->second;
        for (int k = 0; k < 3; ++k) {
            const double f = d->frac[3 * i + k];
            double w = f - std::floor(f);   // numpy.mod(f, 1) for finite f
            if (w >= 1.0) w = 0.0;
            frac[3 * i + k] = w;
        }
    }
    s.n_types = (int)ids.size();
    {
        uint64_t hsh = 1469598103934665603ull;
        auto mix = [&hsh](const void *p, size_t n) {
            const unsigned char *c = static_cast<const unsigned char *>(p);
            for (size_t i = 0; i < n; ++i) hsh = (hsh ^ c[i]) * 1099511628211ull;
        };
        mix(h, 9 * sizeof(double));
        mix(&d->cutoff, sizeof(double));
        mix(&s.n_atoms, sizeof(int));
        mix(frac.data(), frac.size() * sizeof(double));
        mix(type.data(), type.size() * sizeof(int));
        std::vector<std::pair<double, double>> by_id(ids.size());
        for (auto &kv : ids) by_id[kv.second] = kv.first;
        mix(by_id.data(), by_id.size() * sizeof(by_id[0]));
        s.frame_hash = hsh;
    }
    if (s.n_types > kMaxTypes) {
        delete handle;
        return fail(VEXT_ERR_CAPACITY, "%d distinct framework (sigma, epsilon) pairs; limit %d",
                    (int)ids.size(), kMaxTypes);
    }
    std::vector<float4> tf(s.n_types);
    s.h_td.assign(4 * (size_t)s.n_types, 0.0);
    for (auto &kv : ids) {
        const int t = kv.second;
        const double ms = (kv.first.first + d->guest_sigma) / 2;
        const double me = std::sqrt(kv.first.second * d->guest_epsilon);
        const double s6 = std::pow(ms, 6);
        const double c12 = 4 * me * (s6 * s6);
        const double c6 = 4 * me * s6;
        const double cut6 = std::pow(ms / d->cutoff, 6);
        const double shift = -4 * me * (cut6 * cut6 - cut6);
        const double floor2 = (.1 * ms) * (.1 * ms);
        s.h_td[4 * t + 0] = c12;
        s.h_td[4 * t + 1] = c6;
        s.h_td[4 * t + 2] = shift;
        s.h_td[4 * t + 3] = floor2;
        tf[t] = make_float4((float)c12, (float)c6, (float)shift, (float)floor2);
    }
    cudaError_t err = cudaSuccess;
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && err == cudaSuccess) err = e;
    };
    chk(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
    chk(cudaStreamCreateWithFlags(&s.aux, cudaStreamNonBlocking));
    for (auto &e : s.ev) chk(cudaEventCreate(&e));
    chk(cudaMalloc(&s.d_frac, sizeof(double) * frac.size()));
    chk(cudaMalloc(&s.d_type, sizeof(int) * type.size()));
    chk(cudaMalloc(&s.d_tf, sizeof(float4) * tf.size()));
    chk(cudaMalloc(&s.d_td, sizeof(double) * s.h_td.size()));
    chk(cudaMalloc(&s.d_status, sizeof(int)));
    if (err == cudaSuccess) {
        chk(cudaMemcpy(s.d_frac, frac.data(), sizeof(double) * frac.size(), cudaMemcpyHostToDevice));
        chk(cudaMemcpy(s.d_type, type.data(), sizeof(int) * type.size(), cudaMemcpyHostToDevice));
        chk(cudaMemcpy(s.d_tf, tf.data(), sizeof(float4) * tf.size(), cudaMemcpyHostToDevice));
        chk(cudaMemcpy(s.d_td, s.h_td.data(), sizeof(double) * s.h_td.size(),
                       cudaMemcpyHostToDevice));
        chk(cudaMemset(s.d_status, 0, sizeof(int)));
    }
    if (err != cudaSuccess) {
        delete handle;
        return fail(VEXT_ERR_CUDA, "system upload failed: %s", cudaGetErrorString(err));
    }
    *out = handle;
    return 0;
}

extern "C" int vext_system_invalidate(vext_system h) {
    if (!h) return fail(VEXT_ERR_ARGUMENT, "null system");
    std::lock_guard<std::mutex> guard(h->sys.lock);
    for (RegionSet *rs : h->sys.sets) rs->stale = true;
    h->sys.drop_adjoint_batch();
    return 0;
}

extern "C" int vext_last_timings(vext_system h, double *list_ms, double *near_ms,
                                 double *far_ms, double *epilogue_ms) {
    if (!h) return fail(VEXT_ERR_ARGUMENT, "null system");
    System &s = h->sys;
    std::lock_guard<std::mutex> guard(s.lock);
    float a = 0, b = 0, c = 0, d = 0;
    if (s.list_timed) {
        VEXT_CUDA(cudaEventSynchronize(s.ev[4]));
        VEXT_CUDA(cudaEventElapsedTime(&a, s.ev[3], s.ev[4]));
    }
    if (s.timed) {
        VEXT_CUDA(cudaEventSynchronize(s.ev[2]));
        if (s.split_timed) {
            VEXT_CUDA(cudaEventElapsedTime(&b, s.ev[0], s.ev[5]));
            VEXT_CUDA(cudaEventElapsedTime(&c, s.ev[5], s.ev[1]));
        } else {
            VEXT_CUDA(cudaEventElapsedTime(&b, s.ev[0], s.ev[1]));
        }
        VEXT_CUDA(cudaEventElapsedTime(&d, s.ev[1], s.ev[2]));
    }
    if (list_ms) *list_ms = s.list_timed ? a : 0.0;
    if (near_ms) *near_ms = b;
    if (far_ms) *far_ms = c;
    if (epilogue_ms) *epilogue_ms = d;
    s.list_timed = false;
    return 0;
}

extern "C" int vext_system_destroy(vext_system sys) {
    if (!sys) return 0;
    int dev = 0;
    cudaGetDevice(&dev);
    const int own = sys->sys.device;
    if (dev != own) cudaSetDevice(own);
    delete sys;
    if (dev != own) cudaSetDevice(dev);
    return 0;
}
