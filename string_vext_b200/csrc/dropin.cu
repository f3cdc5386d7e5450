// Drop-in `evaluate_reused_neighbors` (reference: native/vext/kernel.cpp:5-45,
// bound by src/string_vext/native.py:18-22 and called at native.py:60-64).
//
// Same arguments, host buffers, output [center][axis] FP64 and return codes
// 0-4.  The validation that yields codes 1-3 runs on the host in the
// reference's order before any device work; the sum runs on the device.
// Each thread owns one (center, director) pose and accumulates exactly as the
// reference does: one running FP64 sum, site 0 then site 1, neighbours in CSR
// order, every operation a separately rounded IEEE op (__dmul_rn, __dadd_rn,
// __ddiv_rn: no FMA contraction) -- so the output is bit-identical to the
// reference kernel compiled for x86-64.  Non-finite energies (code 4) are
// detected on the host in (center, axis) order, and the output is written
// only for the poses the reference would have written before returning.
//
// Device copies of the images and per-image coefficients are cached between
// calls (the reference driver passes the same arrays for every 512-center
// batch); the cache is keyed on the array contents, not only the pointers.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "dropin.cuh"

namespace vext {

__global__ void csr_kernel(CsrArgs a) {
    __shared__ double rec[kCsrChunk * 7];
    const int c = blockIdx.x;
    const long long lo = a.starts[c], hi = a.starts[c + 1];
    for (int a0 = 0; a0 < a.n_axes; a0 += blockDim.x) {
        const int ax = a0 + threadIdx.x;
        const bool valid = ax < a.n_axes;
        const int axc = valid ? ax : 0;
        double energy = 0.0;
        for (int site = 0; site < 2; ++site) {
            const double off = site ? a.off1 : a.off0;
            const double x = dadd(a.centers[3 * c], dmul(off, a.axes[3 * axc]));
            const double y = dadd(a.centers[3 * c + 1], dmul(off, a.axes[3 * axc + 1]));
            const double z = dadd(a.centers[3 * c + 2], dmul(off, a.axes[3 * axc + 2]));
            for (long long n0 = lo; n0 < hi; n0 += kCsrChunk) {
                const int len = (int)min((long long)kCsrChunk, hi - n0);
                __syncthreads();
                for (int t = threadIdx.x; t < len; t += blockDim.x) {
                    const double *r = a.images8 + 8 * (long long)a.indices[n0 + t];
#pragma unroll
                    for (int k = 0; k < 7; ++k) rec[7 * t + k] = r[k];
                }
                __syncthreads();
                for (int t = 0; t < len; ++t) {
                    const double *r = rec + 7 * t;
                    const double dx = dsub(x, r[0]), dy = dsub(y, r[1]), dz = dsub(z, r[2]);
                    const double d2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
                    if (d2 >= a.cutoff2) continue;
                    const double s2 = d2 < r[6] ? r[6] : d2;
                    const double i2 = __ddiv_rn(1.0, s2);
                    const double i6 = dmul(dmul(i2, i2), i2);
                    const double term =
                        dadd(dsub(dmul(dmul(r[3], i6), i6), dmul(r[4], i6)), r[5]);
                    energy = dadd(energy, term);
                }
            }
        }
        if (valid) a.out[(long long)c * a.n_axes + ax] = energy;
    }
}

struct DropinContext {
    std::mutex lock;
    int device = -1;
    cudaStream_t stream = nullptr;
    // cached images (host copy for change detection + device records)
    std::vector<double> h_images, h_c12, h_c6, h_shift, h_floor2;
    double *d_images8 = nullptr;
    size_t images_cap = 0;
    // per-call buffers
    double *d_centers = nullptr, *d_axes = nullptr, *d_out = nullptr;
    size_t centers_cap = 0, axes_cap = 0, out_cap = 0;
    long long *d_starts = nullptr;
    size_t starts_cap = 0;
    int *d_indices = nullptr;
    size_t indices_cap = 0;
    double *h_out = nullptr;   // pinned staging
    size_t h_out_cap = 0;
    std::vector<long long> rebased;
};

static DropinContext g_ctx;

static bool same(const std::vector<double> &v, const double *p, size_t n) {
    return v.size() == n && std::memcmp(v.data(), p, n * sizeof(double)) == 0;
}

static int upload_images(DropinContext &cx, int n_images, const double *images,
                         const double *c12, const double *c6, const double *shift,
                         const double *floor2) {
    const size_t n = (size_t)n_images;
    if (cx.d_images8 && same(cx.h_images, images, 3 * n) && same(cx.h_c12, c12, n) &&
        same(cx.h_c6, c6, n) && same(cx.h_shift, shift, n) && same(cx.h_floor2, floor2, n))
        return 0;
    cx.h_images.assign(images, images + 3 * n);
    cx.h_c12.assign(c12, c12 + n);
    cx.h_c6.assign(c6, c6 + n);
    cx.h_shift.assign(shift, shift + n);
    cx.h_floor2.assign(floor2, floor2 + n);
    std::vector<double> rec(8 * n);
    for (size_t i = 0; i < n; ++i) {
        rec[8 * i + 0] = images[3 * i];
        rec[8 * i + 1] = images[3 * i + 1];
        rec[8 * i + 2] = images[3 * i + 2];
        rec[8 * i + 3] = c12[i];
        rec[8 * i + 4] = c6[i];
        rec[8 * i + 5] = shift[i];
        rec[8 * i + 6] = floor2[i];
        rec[8 * i + 7] = 0.0;
    }
    VEXT_TRY(ensure_capacity(cx.d_images8, cx.images_cap, 8 * n));
    VEXT_CUDA(cudaMemcpyAsync(cx.d_images8, rec.data(), sizeof(double) * 8 * n,
                              cudaMemcpyHostToDevice, cx.stream));
    VEXT_CUDA(cudaStreamSynchronize(cx.stream));   // `rec` is pageable and goes out of scope
    return 0;
}

}  // namespace vext

using namespace vext;

extern "C" int evaluate_reused_neighbors(int n_centers, int n_axes, int n_images, double cutoff2,
                                         const double *centers, const double *axes,
                                         const double *images, const double *offsets,
                                         const double *coeff12, const double *coeff6,
                                         const double *shift, const double *floor2,
                                         const int64_t *starts, const int32_t *indices,
                                         double *output) {
    // code 1 exactly as kernel.cpp:11-12 (a NaN cutoff2 passes, as there)
    if (n_centers < 0 || n_axes < 1 || n_images < 1 || cutoff2 <= 0) return 1;
    if (n_centers == 0) return 0;
    // codes 2/3 in the reference's order: center by center, starts first,
    // then every neighbour index of that center.
    int bad_center = n_centers, bad_code = 0;
    if (starts[0] < 0) {
        bad_center = 0;
        bad_code = 2;
    }
    for (int c = 0; c < bad_center; ++c) {
        if (starts[c] > starts[c + 1]) {
            bad_center = c;
            bad_code = 2;
            break;
        }
        for (int64_t k = starts[c]; k < starts[c + 1]; ++k)
            if (indices[k] < 0 || indices[k] >= n_images) {
                bad_center = c;
                bad_code = 3;
                break;
            }
        if (bad_code) break;
    }
    const int n_eval = bad_center;   // centers the reference evaluates before any 2/3
    if (n_eval == 0) return bad_code;
    DropinContext &cx = g_ctx;
    std::lock_guard<std::mutex> guard(cx.lock);
    int dev = 0;
    VEXT_CUDA(cudaGetDevice(&dev));
    if (cx.device != dev || !cx.stream) {
        // First call, or the caller switched devices: start a fresh cache on
        // this device (buffers of the previous device are released there).
        if (cx.stream) {
            int cur = dev;
            cudaSetDevice(cx.device);
            cudaStreamDestroy(cx.stream);
            for (void *p : {(void *)cx.d_images8, (void *)cx.d_centers, (void *)cx.d_axes,
                            (void *)cx.d_out, (void *)cx.d_starts, (void *)cx.d_indices})
                cudaFree(p);
            cudaSetDevice(cur);
        }
        cx.d_images8 = cx.d_centers = cx.d_axes = cx.d_out = nullptr;
        cx.d_starts = nullptr;
        cx.d_indices = nullptr;
        cx.images_cap = cx.centers_cap = cx.axes_cap = cx.out_cap = 0;
        cx.starts_cap = cx.indices_cap = 0;
        cx.h_images.clear();
        cx.device = dev;
        VEXT_CUDA(cudaStreamCreateWithFlags(&cx.stream, cudaStreamNonBlocking));
    }
    if (n_eval > 0) {
        VEXT_TRY(upload_images(cx, n_images, images, coeff12, coeff6, shift, floor2));
        const long long base = starts[0];
        const long long nnz = starts[n_eval] - base;
        cx.rebased.resize((size_t)n_eval + 1);
        for (int c = 0; c <= n_eval; ++c) cx.rebased[c] = starts[c] - base;
        const size_t n_out = (size_t)n_eval * n_axes;
        VEXT_TRY(ensure_capacity(cx.d_centers, cx.centers_cap, 3 * (size_t)n_eval));
        VEXT_TRY(ensure_capacity(cx.d_axes, cx.axes_cap, 3 * (size_t)n_axes));
        VEXT_TRY(ensure_capacity(cx.d_out, cx.out_cap, n_out));
        VEXT_TRY(ensure_capacity(cx.d_starts, cx.starts_cap, (size_t)n_eval + 1));
        VEXT_TRY(ensure_capacity(cx.d_indices, cx.indices_cap, (size_t)(nnz > 0 ? nnz : 1)));
        if (cx.h_out_cap < n_out) {
            if (cx.h_out) cudaFreeHost(cx.h_out);
            cx.h_out = nullptr;
            cx.h_out_cap = 0;
            VEXT_CUDA(cudaMallocHost(&cx.h_out, sizeof(double) * n_out));
            cx.h_out_cap = n_out;
        }
        cudaStream_t st = cx.stream;
        VEXT_CUDA(cudaMemcpyAsync(cx.d_centers, centers, sizeof(double) * 3 * n_eval,
                                  cudaMemcpyHostToDevice, st));
        VEXT_CUDA(cudaMemcpyAsync(cx.d_axes, axes, sizeof(double) * 3 * n_axes,
                                  cudaMemcpyHostToDevice, st));
        VEXT_CUDA(cudaMemcpyAsync(cx.d_starts, cx.rebased.data(), sizeof(long long) * (n_eval + 1),
                                  cudaMemcpyHostToDevice, st));
        if (nnz > 0)
            VEXT_CUDA(cudaMemcpyAsync(cx.d_indices, indices + base, sizeof(int) * nnz,
                                      cudaMemcpyHostToDevice, st));
        CsrArgs a;
        a.n_centers = n_eval;
        a.n_axes = n_axes;
        a.cutoff2 = cutoff2;
        a.centers = cx.d_centers;
        a.axes = cx.d_axes;
        a.images8 = cx.d_images8;
        a.off0 = offsets[0];
        a.off1 = offsets[1];
        a.starts = cx.d_starts;
        a.indices = cx.d_indices;
        a.out = cx.d_out;
        const int threads = n_axes >= 128 ? 128 : ((n_axes + 31) / 32) * 32;
        csr_kernel<<<n_eval, threads, 0, st>>>(a);
        VEXT_CUDA(cudaGetLastError());
        VEXT_CUDA(cudaMemcpyAsync(cx.h_out, cx.d_out, sizeof(double) * n_out,
                                  cudaMemcpyDeviceToHost, st));
        VEXT_CUDA(cudaStreamSynchronize(st));
        // code 4 at the first non-finite pose in (center, axis) order; the
        // reference writes every pose before it and none after.
        for (size_t i = 0; i < n_out; ++i)
            if (!std::isfinite(cx.h_out[i])) {
                std::memcpy(output, cx.h_out, sizeof(double) * i);
                return 4;
            }
        std::memcpy(output, cx.h_out, sizeof(double) * n_out);
    }
    return bad_code;
}
