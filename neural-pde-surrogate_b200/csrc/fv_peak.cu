// FP64 pipe peak of the current device, measured: the denominator of the FP64 roofline that the
// finite-volume kernels are reported against (the HBM and bf16 peaks come from elsewhere; nothing
// measures the FP64 pipe for us).  Eight independent DFMA chains per thread keep the pipe full.
#include <cuda_runtime.h>

#include "../../include/fv.h"

namespace {

constexpr int kChains = 8, kIters = 2048, kThreads = 256;

__global__ void __launch_bounds__(kThreads) dfma_peak_kernel(double* out, double a, double b) {
    double x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-9 + k;
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == 12345.678) out[0] = s;  // keeps the chains alive; practically never taken
}

}  // namespace

extern "C" int fv_fp64_peak(double* dfma_per_second) {
    if (!dfma_per_second) return FV_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FV_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return FV_ERR_CUDA;
    double* d = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return FV_ERR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8;
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        dfma_peak_kernel<<<blocks, kThreads>>>(d, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;  // first launch is warm-up
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (err != cudaSuccess) return FV_ERR_CUDA;
    *dfma_per_second = double(blocks) * kThreads * kChains * kIters / (best * 1e-3);
    return FV_OK;
}
