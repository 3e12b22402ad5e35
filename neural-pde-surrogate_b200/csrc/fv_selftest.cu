// Self-tests of the library's device code: the bounded waits, and the division sequences of the
// stage kernels against IEEE division (second half of this file).
//
// Bounded waits.  Every asynchronous copy (the stage kernels' TMA halo boxes) and
// every tensor-core batch (the correction network's convolutions) of this library is waited for with
// tc::mbar_wait_bounded, which gives up after a time limit, records an error for the host and lets
// the kernel return instead of spinning forever.  This entry point runs that same wait on an
// mbarrier that nothing ever arrives at, with a short limit, so that a test can watch the give-up path
// end by itself and report, and check that the context is still usable afterwards.
#include <cuda_runtime.h>

#include <climits>

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

// ---- the persistent stepper's waits ---------------------------------------------------------------
// The stepper's two waits -- for a step's publication and for the neighbour tiles' flags -- run here
// against control blocks and a flag that nothing will ever publish, each with a 10 ms limit: each
// must give up and record FV_ERR_TIMEOUT in its control block.  A second CTA waits on the flags'
// control block with the default 1 s limit and must leave as soon as it sees that status.
#include "fv_stepper.cuh"

namespace {

// Device memory of the test: two control blocks, then one flag (never set), the dependency list of
// a single tile on itself (offsets {0, 1}, index {0}) and three outcomes.
struct WaitTest {
    fv::FvCtrl c[2];
    unsigned flag;
    int dep[3];
    int outcome[3];
};

__global__ void stepper_wait_selftest_kernel(WaitTest* w) {
    const fv::StepperTiles st{&w->flag, &w->flag, w->dep, w->dep + 2, 1, 1, 0};
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) w->outcome[0] = fv::wait_complete(&w->c[0], 5, 10000000ull) ? 1 : 2;
        __syncwarp();
        const bool ok = fv::wait_flags(&w->c[1], &w->flag, st, 0, 7u, 10000000ull);
        if (threadIdx.x == 0) w->outcome[1] = ok ? 1 : 2;
    } else {
        const uint64_t t0 = tc::globaltimer_ns();
        const bool ok = fv::wait_flags(&w->c[1], &w->flag, st, 0, 7u);
        if (threadIdx.x == 0) w->outcome[2] = ok ? 1 : (tc::globaltimer_ns() - t0 < 500000000ull ? 2 : 3);
    }
}

}  // namespace

extern "C" int fv_stepper_wait_selftest(void) {
    WaitTest h{};
    for (auto& c : h.c) {
        c.complete = -1;       // no step published
        c.stop = LLONG_MAX;    // and none known not to run
    }
    h.dep[1] = 1;              // offsets {0, 1}, index {0}
    WaitTest* d = nullptr;
    if (cudaMalloc(&d, sizeof(WaitTest)) != cudaSuccess) return FV_ERR_CUDA;
    cudaError_t e = cudaMemcpy(d, &h, sizeof h, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        stepper_wait_selftest_kernel<<<2, 32>>>(d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return FV_ERR_CUDA;
    const bool gave_up = h.outcome[0] == 2 && h.outcome[1] == 2 && h.outcome[2] == 2;
    return (gave_up && h.c[0].status == FV_ERR_TIMEOUT && h.c[1].status == FV_ERR_TIMEOUT) ? FV_ERR_TIMEOUT
                                                                                           : FV_ERR_STATE;
}

// ---- the divisions of the stage kernels against IEEE division -------------------------------------
// The stage kernels replace IEEE a / b by cheaper sequences where those give the same quotient:
// div_gm1 (p / (GAMMA - 1)), div_z (zero numerators), div_back (a face state's velocity after the
// to_conserved / to_primitive round trip), and, in the tolerance build only, fdiv at every general
// division site.  These entry points run each sequence on the GPU so that tests can compare it with
// IEEE division (__ddiv_rn) bit for bit: on given operands, and on billions of operands drawn on
// the device.
#include "fv_physics.cuh"

namespace {

__device__ __forceinline__ double eval_kind(int kind, double a, double b) {
    switch (kind) {
    case FV_DIV_GM1: return fv::div_gm1(a);
    case FV_DIV_ZERO: return fv::div_z(a, b);
    case FV_DIV_BACK: return fv::div_back(__dmul_rn(a, b), a, b);
    default: return fv::fdiv(a, b);
    }
}

// The IEEE quotient each kind stands for.
__device__ __forceinline__ double ieee_kind(int kind, double a, double b) {
    switch (kind) {
    case FV_DIV_GM1: return __ddiv_rn(a, fv::GM1);
    case FV_DIV_BACK: return __ddiv_rn(__dmul_rn(a, b), a);
    default: return __ddiv_rn(a, b);
    }
}

__global__ void division_kind_kernel(int kind, int n, const double* __restrict__ a, const double* __restrict__ b,
                                     double* __restrict__ q) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        q[k] = eval_kind(kind, a[k], b ? b[k] : 0.0);
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// A random double: r supplies the mantissa, c the class.  Mostly normal numbers with exponents within
// +-spread of 1 (the range the solver sees), some across the whole exponent range, and the edge
// patterns: zeros, subnormals, infinities, and all-ones / zero / single-bit mantissas.
__device__ double draw(uint64_t r, uint64_t c, int spread, int zero_in_64) {
    const uint64_t sign = (c >> 63) << 63;
    const int cls = int(c & 63u);
    uint64_t mant = r & 0xfffffffffffffull;
    const int mcls = int((c >> 6) & 15u);
    if (mcls == 0) mant = 0xfffffffffffffull;
    else if (mcls == 1) mant = 0;
    else if (mcls == 2) mant = 1ull << (r % 52);
    int e;
    if (cls < zero_in_64) return __longlong_as_double((long long)sign);  // +-0
    if (cls == 62) return __longlong_as_double((long long)(sign | mant | 1ull));  // subnormal
    if (cls == 63) return __longlong_as_double((long long)(sign | (0x7ffull << 52)));  // +-inf
    if (cls >= 54) e = 1 + int((c >> 10) % 2046u);  // anywhere in the normal range
    else e = 1023 - spread + int((c >> 10) % uint64_t(2 * spread + 1));
    return __longlong_as_double((long long)(sign | (uint64_t(e) << 52) | mant));
}

__device__ __forceinline__ long long ordered(double x) {
    const long long i = __double_as_longlong(x);
    return i < 0 ? (long long)(0x8000000000000000ull - (unsigned long long)i) : i;
}

__global__ void division_sweep_kernel(int kind, long long n, unsigned long long seed, unsigned long long* mism,
                                      unsigned long long* max_ulps) {
    unsigned long long count = 0, worst = 0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const uint64_t base = splitmix64(seed ^ (uint64_t(k) * 0x2545f4914f6cdd1dull));
        const uint64_t r0 = splitmix64(base + 1), r1 = splitmix64(base + 2), r2 = splitmix64(base + 3),
                       r3 = splitmix64(base + 4);
        double a, b;
        if (kind == FV_DIV_BACK) {  // a = rho: mostly positive densities; b = u: velocities, some zero
            a = fabs(draw(r0, r1, 40, 1));
            if ((r1 & 0xf00000ull) == 0) a = -a;  // 1 in 16: a negative density (the guarded path)
            b = draw(r2, r3, 80, 4);
        } else {
            a = draw(r0, r1, 80, kind == FV_DIV_ZERO ? 16 : 1);
            b = draw(r2, r3, 80, 1);
        }
        const double q = eval_kind(kind, a, b), ref = ieee_kind(kind, a, b);
        const bool qn = q != q, rn = ref != ref;
        if (qn && rn) continue;  // both NaN
        const long long d = (qn || rn) ? LLONG_MAX : llabs(ordered(q) - ordered(ref));
        if (__double_as_longlong(q) != __double_as_longlong(ref)) {
            ++count;
            if ((unsigned long long)d > worst) worst = (unsigned long long)d;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        count += __shfl_xor_sync(0xffffffffu, count, o);
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, worst, o);
        worst = w > worst ? w : worst;
    }
    if ((threadIdx.x & 31) == 0) {
        if (count) atomicAdd(mism, count);
        if (worst) atomicMax(max_ulps, worst);
    }
}

}  // namespace

int fv_internal_set_error(int code, const char* msg);  // fv_api.cu: sets fv_last_error()

extern "C" int fv_eval_division_kind(int kind, int n, const double* a, const double* b, double* q) {
    if (kind < FV_DIV_GENERAL || kind > FV_DIV_BACK)
        return fv_internal_set_error(FV_ERR_ARG, "fv_eval_division_kind: unknown kind");
    if (n < 0 || (n > 0 && (!a || !q || (!b && kind != FV_DIV_GM1))))
        return fv_internal_set_error(FV_ERR_ARG, "fv_eval_division_kind: bad arguments");
    if (n == 0) return FV_OK;
    double* d = nullptr;
    const size_t bytes = size_t(n) * sizeof(double);
    if (cudaMalloc(&d, 3 * bytes) != cudaSuccess) return fv_internal_set_error(FV_ERR_CUDA, "cudaMalloc failed");
    cudaError_t e = cudaMemcpy(d, a, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && b) e = cudaMemcpy(d + n, b, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        division_kind_kernel<<<(n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184, 256>>>(kind, n, d, b ? d + n : nullptr,
                                                                                      d + 2 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(q, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fv_internal_set_error(FV_ERR_CUDA, cudaGetErrorString(e));
    return FV_OK;
}

extern "C" int fv_division_sweep(int kind, long long n, unsigned long long seed, long long* mismatches,
                                 long long* max_ulps) {
    if (kind < FV_DIV_GENERAL || kind > FV_DIV_BACK || n < 0 || !mismatches)
        return fv_internal_set_error(FV_ERR_ARG, "fv_division_sweep: bad arguments");
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(unsigned long long)) != cudaSuccess)
        return fv_internal_set_error(FV_ERR_CUDA, "cudaMalloc failed");
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaMemset(d, 0, sizeof(h));
    if (e == cudaSuccess && n > 0) {
        division_sweep_kernel<<<148 * 8, 256>>>(kind, n, seed, d, d + 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fv_internal_set_error(FV_ERR_CUDA, cudaGetErrorString(e));
    *mismatches = (long long)h[0];
    if (max_ulps) *max_ulps = (long long)h[1];
    return FV_OK;
}
