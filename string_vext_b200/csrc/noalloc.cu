// evaluate_reused_neighbors_noalloc: the drop-in CSR pair sum for callers
// that must not allocate device memory.
//
// Who needs this: plug-ins hosted by a runtime that owns the GPU memory
// budget and forbids allocations of its own (fixed-pool inference or
// simulation servers, MPS clients with hard memory limits, applications that
// hand out device memory only through their own allocator), and real-time
// loops where an allocation's implicit device synchronisation is
// unacceptable.  The regular entry point grows cached device buffers with
// cudaMalloc on demand; this one never calls cudaMalloc, cudaFree,
// cudaMallocHost or any allocating library routine, and uses no host heap.
//
// Its scratch is g_noalloc_scratch below, a file-scope device array of
// kNoAllocBytes (64 MiB) that every GPU loading this library holds until the
// process exits.  A batch fits when
//   120 n_images + 24 (n_centers + n_axes) + 8 (n_centers + 1) + 4 nnz
//   + 8 n_centers n_axes   (+ 256-byte alignment per part)  <=  64 MiB,
// e.g. 165,000 images, 512 centers x 64 directors and 800,000 neighbours
// take about 23 MiB.
// Larger batches are rejected with VEXT_ERR_CAPACITY before anything is
// copied to the device (the host checks of codes 2 and 3 come first and read
// starts and indices).
//
// In host code `g_noalloc_scratch` only names a host-side stand-in; the
// device address comes from cudaGetSymbolAddress with the calling thread's
// current device, checked and passed to the kernels.  The first call on a
// device also loads the module holding the array there.  The address is
// looked up again on every call (a lookup, not an allocation), so a device
// reset between calls cannot leave a stale address behind.  Every call
// reuses the same array and leaves the previous call's contents in it;
// nothing in it has to start at zero (each call writes every byte it reads
// before reading it; the one word that must start from a known value, the
// first non-finite index, is set by a copy each call).  Calls are serialised
// by a process-wide mutex and complete before returning, so calls from this
// process never overlap on the GPU; calls that did overlap on the GPU (from
// another process sharing the module, or by bypassing the mutex) would race
// on the array.
//
// Semantics are those of evaluate_reused_neighbors (same arguments, host
// buffers, return codes 0-4 in the reference's order, bit-identical FP64
// output, only the prefix the reference writes on code 4), plus
// VEXT_ERR_CAPACITY.  Work is issued on the calling thread's per-thread
// default stream, and the call returns when it is done.
#include <cmath>
#include <mutex>

#include "dropin.cuh"

namespace vext {

constexpr size_t kNoAllocBytes = 64ull << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_lock;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device address of the scratch array on the current device.
int scratch_address(unsigned char **out) {
    void *p = nullptr;
    VEXT_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return fail(VEXT_ERR_CUDA, "no device address for the no-alloc scratch array");
    *out = static_cast<unsigned char *>(p);
    return 0;
}

// Pack the per-image arrays into the 8-double records csr_kernel reads and
// rebase the CSR starts to 0.  One thread per image / center.
__global__ void noalloc_pack_kernel(int n_images, const double *images, const double *c12,
                                    const double *c6, const double *shift,
                                    const double *floor2, double *rec, int n_starts,
                                    long long *starts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_images) {
        double *r = rec + 8 * (long long)i;
        r[0] = images[3 * (long long)i];
        r[1] = images[3 * (long long)i + 1];
        r[2] = images[3 * (long long)i + 2];
        r[3] = c12[i];
        r[4] = c6[i];
        r[5] = shift[i];
        r[6] = floor2[i];
        r[7] = 0.0;
    }
    if (blockIdx.x == 0)   // starts[0] itself is zeroed by the next kernel
        for (int c = n_starts - 1 - threadIdx.x; c >= 1; c -= blockDim.x)
            starts[c] -= starts[0];
}

__global__ void noalloc_zero_first_kernel(long long *starts) { starts[0] = 0; }

// First non-finite output in (center, axis) order, or n if none.
__global__ void noalloc_first_nonfinite_kernel(const double *out, long long n,
                                               unsigned long long *first) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (!isfinite(out[i])) atomicMin(first, (unsigned long long)i);
}

}  // namespace
}  // namespace vext

using namespace vext;

extern "C" int evaluate_reused_neighbors_noalloc(int n_centers, int n_axes, int n_images,
                                                 double cutoff2, const double *centers,
                                                 const double *axes, const double *images,
                                                 const double *offsets, const double *coeff12,
                                                 const double *coeff6, const double *shift,
                                                 const double *floor2, const int64_t *starts,
                                                 const int32_t *indices, double *output) {
    if (n_centers < 0 || n_axes < 1 || n_images < 1 || cutoff2 <= 0) return 1;
    if (n_centers == 0) return 0;
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
    const int n_eval = bad_center;
    if (n_eval == 0) return bad_code;
    const long long base = starts[0];
    const long long nnz = starts[n_eval] - base;
    const size_t n_out = (size_t)n_eval * n_axes;
    // layout of the scratch array (every part 256-byte aligned)
    const size_t o_rec = 0;
    const size_t o_img = o_rec + align256(64 * (size_t)n_images);
    const size_t o_coef = o_img + align256(24 * (size_t)n_images);
    const size_t o_cent = o_coef + 4 * align256(8 * (size_t)n_images);
    const size_t o_axes = o_cent + align256(24 * (size_t)n_eval);
    const size_t o_start = o_axes + align256(24 * (size_t)n_axes);
    const size_t o_idx = o_start + align256(8 * ((size_t)n_eval + 1));
    const size_t o_out = o_idx + align256(4 * (size_t)(nnz > 0 ? nnz : 1));
    const size_t o_first = o_out + align256(8 * n_out);
    const size_t total = o_first + 256;
    if (total > kNoAllocBytes)
        return fail(VEXT_ERR_CAPACITY,
                    "evaluate_reused_neighbors_noalloc: batch needs %zu bytes of scratch, "
                    "limit %zu (n_images %d, centers %d, directors %d, neighbours %lld)",
                    total, kNoAllocBytes, n_images, n_eval, n_axes, nnz);
    std::lock_guard<std::mutex> guard(g_noalloc_lock);
    unsigned char *s = nullptr;
    VEXT_TRY(scratch_address(&s));
    cudaStream_t st = cudaStreamPerThread;
    double *rec = reinterpret_cast<double *>(s + o_rec);
    double *d_img = reinterpret_cast<double *>(s + o_img);
    double *d_c12 = reinterpret_cast<double *>(s + o_coef);
    double *d_c6 = reinterpret_cast<double *>(s + o_coef + align256(8 * (size_t)n_images));
    double *d_sh = reinterpret_cast<double *>(s + o_coef + 2 * align256(8 * (size_t)n_images));
    double *d_fl = reinterpret_cast<double *>(s + o_coef + 3 * align256(8 * (size_t)n_images));
    double *d_cent = reinterpret_cast<double *>(s + o_cent);
    double *d_axes = reinterpret_cast<double *>(s + o_axes);
    long long *d_start = reinterpret_cast<long long *>(s + o_start);
    int *d_idx = reinterpret_cast<int *>(s + o_idx);
    double *d_out = reinterpret_cast<double *>(s + o_out);
    unsigned long long *d_first = reinterpret_cast<unsigned long long *>(s + o_first);
    const size_t ni = (size_t)n_images;
    VEXT_CUDA(cudaMemcpyAsync(d_img, images, 24 * ni, cudaMemcpyHostToDevice, st));
    VEXT_CUDA(cudaMemcpyAsync(d_c12, coeff12, 8 * ni, cudaMemcpyHostToDevice, st));
    VEXT_CUDA(cudaMemcpyAsync(d_c6, coeff6, 8 * ni, cudaMemcpyHostToDevice, st));
    VEXT_CUDA(cudaMemcpyAsync(d_sh, shift, 8 * ni, cudaMemcpyHostToDevice, st));
    VEXT_CUDA(cudaMemcpyAsync(d_fl, floor2, 8 * ni, cudaMemcpyHostToDevice, st));
    VEXT_CUDA(cudaMemcpyAsync(d_cent, centers, 24 * (size_t)n_eval, cudaMemcpyHostToDevice, st));
    VEXT_CUDA(cudaMemcpyAsync(d_axes, axes, 24 * (size_t)n_axes, cudaMemcpyHostToDevice, st));
    VEXT_CUDA(cudaMemcpyAsync(d_start, starts, 8 * ((size_t)n_eval + 1), cudaMemcpyHostToDevice,
                              st));
    if (nnz > 0)
        VEXT_CUDA(cudaMemcpyAsync(d_idx, indices + base, 4 * (size_t)nnz, cudaMemcpyHostToDevice,
                                  st));
    const int blocks = (n_images + 255) / 256;
    noalloc_pack_kernel<<<blocks, 256, 0, st>>>(n_images, d_img, d_c12, d_c6, d_sh, d_fl, rec,
                                                n_eval + 1, d_start);
    VEXT_CUDA(cudaGetLastError());
    noalloc_zero_first_kernel<<<1, 1, 0, st>>>(d_start);
    VEXT_CUDA(cudaGetLastError());
    CsrArgs a;
    a.n_centers = n_eval;
    a.n_axes = n_axes;
    a.cutoff2 = cutoff2;
    a.centers = d_cent;
    a.axes = d_axes;
    a.images8 = rec;
    a.off0 = offsets[0];
    a.off1 = offsets[1];
    a.starts = d_start;
    a.indices = d_idx;
    a.out = d_out;
    const int threads = n_axes >= 128 ? 128 : ((n_axes + 31) / 32) * 32;
    csr_kernel<<<n_eval, threads, 0, st>>>(a);
    VEXT_CUDA(cudaGetLastError());
    const unsigned long long none = (unsigned long long)n_out;
    VEXT_CUDA(cudaMemcpyAsync(d_first, &none, sizeof none, cudaMemcpyHostToDevice, st));
    noalloc_first_nonfinite_kernel<<<148, 256, 0, st>>>(d_out, (long long)n_out, d_first);
    VEXT_CUDA(cudaGetLastError());
    unsigned long long first = 0;
    VEXT_CUDA(cudaMemcpyAsync(&first, d_first, sizeof first, cudaMemcpyDeviceToHost, st));
    VEXT_CUDA(cudaStreamSynchronize(st));
    const size_t keep = first < none ? (size_t)first : n_out;
    if (keep)
        VEXT_CUDA(cudaMemcpyAsync(output, d_out, 8 * keep, cudaMemcpyDeviceToHost, st));
    VEXT_CUDA(cudaStreamSynchronize(st));
    if (first < none) return 4;
    return bad_code;
}
