// Diagnostics: the measured non-tensor FP32 roofline of the current device.
//
// fma_peak_kernel runs 16 independent register-resident FFMA chains per
// thread (enough ILP to cover the FMA latency) over a grid of 8 CTAs of 256
// threads per SM; FLOPs = 2 x FMAs.  The result is written to `sink` only if
// it is impossible (NaN), so the chains cannot be optimised away.
#include "internal.cuh"

namespace vext {

__global__ void __launch_bounds__(256) fma_peak_kernel(int iterations, float seed, float *sink) {
    float a[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = seed + 0.001f * (threadIdx.x + k);
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int k = 0; k < 16; ++k) a[k] = fmaf(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += a[k];
    if (s != s) sink[threadIdx.x] = s;
}

// Same with packed FP32x2 FMAs (two FMAs per lane per instruction).
__global__ void __launch_bounds__(256) fma2_peak_kernel(int iterations, float seed, float *sink) {
    float2 a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = make_float2(seed + 0.001f * (threadIdx.x + k), seed - 0.001f * k);
    const float2 m = make_float2(0.999999f, 0.999998f), c = make_float2(1e-7f, 2e-7f);
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] = __ffma2_rn(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k].x + a[k].y;
    if (s != s) sink[threadIdx.x] = s;
}

// Hardware reciprocal throughput (MUFU), 8 independent chains per thread.
__global__ void __launch_bounds__(256) rcp_peak_kernel(int iterations, float seed, float *sink) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + 0.001f * (threadIdx.x + k);
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) asm volatile("rcp.approx.ftz.f32 %0, %0;" : "+f"(a[k]));
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s != s) sink[threadIdx.x] = s;
}

// A staged wait that can never complete: one thread arms the barrier for a
// 16-byte copy that is never issued, then every thread waits through
// mbar_wait_bounded with `polls` as its limit -- the path each staged pair
// kernel takes when a copy does not land.  Nothing is in flight, so the
// barrier is simply invalidated before the CTA exits.
__global__ void wait_timeout_kernel(uint32_t polls, int *status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16);
    __syncthreads();
    mbar_wait_bounded(&bar, 0, status, polls);
    __syncthreads();
    if (threadIdx.x == 0) mbar_inval(&bar);
}

}  // namespace vext

using namespace vext;

extern "C" int vext_check_wait_timeout(int polls) {
    if (polls < 1 || (uint32_t)polls > kWaitLimit)
        return fail(VEXT_ERR_ARGUMENT, "polls must lie in [1, %u]", kWaitLimit);
    int *status = nullptr;
    VEXT_CUDA(cudaMalloc(&status, sizeof(int)));
    int h = DEV_OK;
    cudaError_t err = cudaMemset(status, 0, sizeof(int));
    if (err == cudaSuccess) {
        wait_timeout_kernel<<<1, 32>>>((uint32_t)polls, status);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(status);
    if (err != cudaSuccess)
        return fail(VEXT_ERR_CUDA, "wait_timeout_kernel: %s", cudaGetErrorString(err));
    if (h == DEV_TIMEOUT)
        return fail(VEXT_ERR_TIMEOUT, "a bounded device wait gave up after %d polls", polls);
    return h == DEV_OK ? 0 : fail(VEXT_ERR_CUDA, "unexpected device status %d", h);
}

// ops/s of one probe kernel (kind 0: FFMA, 1: FFMA2 counted as 2 FMAs, 2: RCP)
static int probe(int kind, int iterations, double *ops) {
    int dev = 0, sms = 0;
    VEXT_CUDA(cudaGetDevice(&dev));
    VEXT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float *sink = nullptr;
    VEXT_CUDA(cudaMalloc(&sink, 256 * sizeof(float)));
    cudaEvent_t e0, e1;
    VEXT_CUDA(cudaEventCreate(&e0));
    VEXT_CUDA(cudaEventCreate(&e1));
    const int blocks = sms * 8;
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        const int it = rep ? iterations : iterations / 10 + 1;
        VEXT_CUDA(cudaEventRecord(e0));
        if (kind == 0) fma_peak_kernel<<<blocks, 256>>>(it, 1.0f, sink);
        else if (kind == 1) fma2_peak_kernel<<<blocks, 256>>>(it, 1.0f, sink);
        else rcp_peak_kernel<<<blocks, 256>>>(it, 1.5f, sink);
        VEXT_CUDA(cudaGetLastError());
        VEXT_CUDA(cudaEventRecord(e1));
        VEXT_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        VEXT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep) best = ms < best ? ms : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    const double per_thread = kind == 2 ? 64.0 : 128.0;   // ops per iteration
    *ops = (double)blocks * 256 * iterations * per_thread / (best * 1e-3);
    return 0;
}

extern "C" int vext_measure_pipes(int iterations, double *ffma_per_s, double *ffma2_fma_per_s,
                                  double *rcp_per_s) {
    if (iterations < 1) return fail(VEXT_ERR_ARGUMENT, "bad arguments");
    if (ffma_per_s) VEXT_TRY(probe(0, iterations, ffma_per_s));
    if (ffma2_fma_per_s) VEXT_TRY(probe(1, iterations, ffma2_fma_per_s));
    if (rcp_per_s) VEXT_TRY(probe(2, iterations, rcp_per_s));
    return 0;
}

extern "C" int vext_measure_fp32_peak(int iterations, double *flops_per_second) {
    if (!flops_per_second || iterations < 1) return fail(VEXT_ERR_ARGUMENT, "bad arguments");
    int dev = 0, sms = 0;
    VEXT_CUDA(cudaGetDevice(&dev));
    VEXT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float *sink = nullptr;
    VEXT_CUDA(cudaMalloc(&sink, 256 * sizeof(float)));
    cudaEvent_t e0, e1;
    VEXT_CUDA(cudaEventCreate(&e0));
    VEXT_CUDA(cudaEventCreate(&e1));
    const int blocks = sms * 8;
    fma_peak_kernel<<<blocks, 256>>>(iterations / 10 + 1, 1.0f, sink);   // warm-up
    VEXT_CUDA(cudaGetLastError());
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        VEXT_CUDA(cudaEventRecord(e0));
        fma_peak_kernel<<<blocks, 256>>>(iterations, 1.0f, sink);
        VEXT_CUDA(cudaEventRecord(e1));
        VEXT_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        VEXT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = ms < best ? ms : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    const double fmas = (double)blocks * 256 * iterations * 8 * 16;
    *flops_per_second = 2.0 * fmas / (best * 1e-3);
    return 0;
}
