// Shared host/device helpers of the vext_b200 library: status reporting,
// CUDA error checks, and the mbarrier + 1-D bulk-copy (TMA) primitives used to
// stage region lists into shared memory.  All device waits are bounded: a
// wait that gives up sets a status word the host turns into VEXT_ERR_TIMEOUT.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/vext_b200.h"

namespace vext {

// ---------------------------------------------------------------- host side

void set_error(const char *fmt, ...);   // thread-local message for vext_last_error
int fail(int code, const char *fmt, ...);

#define VEXT_CUDA(call)                                                                 \
    do {                                                                                \
        cudaError_t err_ = (call);                                                      \
        if (err_ != cudaSuccess)                                                        \
            return ::vext::fail(VEXT_ERR_CUDA, "%s failed: %s (%s:%d)", #call,         \
                                cudaGetErrorString(err_), __FILE__, __LINE__);          \
    } while (0)

#define VEXT_TRY(expr)                 \
    do {                               \
        int rc_ = (expr);              \
        if (rc_) return rc_;           \
    } while (0)

// Device status word values (written by kernels, read by the host).
enum : int { DEV_OK = 0, DEV_TIMEOUT = 1, DEV_BAD_LIST = 2, DEV_BAD_INPUT = 3 };

// Upper bound on spin iterations of one mbarrier wait (each try_wait also
// suspends in hardware for a while, so this is about a second of wall time).
constexpr uint32_t kWaitLimit = 1u << 22;

// -------------------------------------------------------------- device side

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait on one phase of an mbarrier.  Returns false (and records
// DEV_TIMEOUT) if the phase did not complete within `limit` polls.
// Once any CTA has recorded a failure, other waits give up at their next
// status poll instead of spinning to their own limit.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *status,
                                                  uint32_t limit = kWaitLimit) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 1023u) == 1023u && *(volatile int *)status != DEV_OK) return false;
    }
    atomicExch(status, DEV_TIMEOUT);
    return false;
}

// Exit path after a failed wait: give copies already issued to this stage
// a bounded time to land (no status poll), so the CTA never exits with a
// bulk copy still writing into its shared memory.
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return;
}

// 1-D bulk copy global -> shared (TMA, no multicast), completion counted on
// `bar` in bytes.  dst/src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// IEEE-exact helpers for the reference-order FP64 sum (no contraction).
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// FP32 reciprocal: hardware approximation refined by one Newton-Raphson step
// r' = r + r (1 - s r) (the classic quadratically convergent iteration).
__device__ __forceinline__ float rcp_nr(float s) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(s));
    const float e = fmaf(-s, r, 1.0f);
    return fmaf(r, e, r);
}

struct Mat3 {
    double m[9];  // row-vector cell: cart_j = sum_k frac_k m[3k + j]
};

// Explicit fused multiply-adds: every kernel that forms a center gets the
// same roundings (the border repair recomputes the far kernel's FP32
// decisions bit for bit from the same center).
__host__ __device__ __forceinline__ void frac_to_cart(const Mat3 &h, double a, double b, double c,
                                                      double &x, double &y, double &z) {
    x = fma(c, h.m[6], fma(b, h.m[3], a * h.m[0]));
    y = fma(c, h.m[7], fma(b, h.m[4], a * h.m[1]));
    z = fma(c, h.m[8], fma(b, h.m[5], a * h.m[2]));
}

}  // namespace vext
