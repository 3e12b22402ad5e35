// Self-test of the bounded waits.  Every asynchronous copy (the stage kernels' TMA halo boxes) and
// every tensor-core batch (the correction network's convolutions) of this library is waited for with
// tc::mbar_wait_bounded, which gives up after a time limit, records an error for the host and lets
// the kernel return instead of spinning forever.  This entry point runs that same wait on an
// mbarrier that nothing ever arrives at, with a short limit, so that a test can watch the give-up path
// end by itself and report, and check that the context is still usable afterwards.
#include <cuda_runtime.h>

#include "../../include/fv.h"
#include "tc_sm100.cuh"

namespace {

__global__ void bounded_wait_selftest_kernel(int* err, int* outcome, unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);  // expects one arrival that never comes
        tc::fence_mbar_init();
    }
    __syncthreads();
    const bool completed = tc::mbar_wait_bounded(&bar, 0, err, limit_ns);
    if (threadIdx.x == 0) *outcome = completed ? 1 : 2;
}

}  // namespace

extern "C" int fv_wait_selftest(void) {
    int* d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(int)) != cudaSuccess) return FV_ERR_CUDA;
    int h[2] = {0, 0};
    cudaError_t e = cudaMemset(d, 0, 2 * sizeof(int));
    if (e == cudaSuccess) {
        bounded_wait_selftest_kernel<<<1, 32>>>(d, d + 1, 10000000ull);  // 10 ms limit
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return FV_ERR_CUDA;
    // the wait must have run out (outcome 2) and recorded it (err 1)
    return (h[0] == 1 && h[1] == 2) ? FV_ERR_TIMEOUT : FV_ERR_STATE;
}
