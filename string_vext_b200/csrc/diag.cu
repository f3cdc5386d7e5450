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

}  // namespace vext

using namespace vext;

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
